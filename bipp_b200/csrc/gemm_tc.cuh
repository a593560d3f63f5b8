// Batched C = L^-1 op(B) on the 5th-generation tensor cores (sm_100a, tcgen05), the two
// products of the reduction C = L^-1 S L^-H of the generalized eigenproblem with a real
// Gram matrix (identity beamforming):
//   T1 = L^-1 S          (op(B) = B)
//   C  = L^-1 T1^H       (op(B) = B^H; C is Hermitian, so T1 L^-T = conj(L^-1 T1^T))
// L^-1 is real, lower triangular, FP32, stored with zeros above its diagonal; B and C
// are complex FP32, column-major. A complex column j of op(B) is two real columns (re,
// im), so one real GEMM of M = 128 rows x N = 128 real columns (64 complex) per CTA
// covers a tile. FP32 accuracy comes from the 3xTF32 split a b ~ a_hi b_hi + a_hi b_lo +
// a_lo b_hi. Threads stage 32 k of A and B per phase into shared memory (canonical
// K-major, no swizzle) and one thread issues the MMAs into a 128 x 128 FP32 accumulator
// in tensor memory; every wait on the MMA completion barrier is bounded, and a timeout
// sets the matrix's status bit (the CTA still frees its tensor memory).
#pragma once

#include "common.cuh"
#include "tc_common.cuh"

namespace bippb200 {

constexpr int kTgThreads = 128;
constexpr int kTgM = 128;                 // rows of C per CTA
constexpr int kTgNC = 64;                 // complex columns of C per CTA
constexpr int kTgN = 2 * kTgNC;           // real columns (MMA N)
constexpr int kTgKP = 32;                 // k per phase
constexpr int kTgSteps = kTgKP / 8;       // MMA K-steps per phase (K = 8 for tf32)
constexpr int kTgAStep = kTgM * 8 * 4;    // bytes of one K-step of A (128 rows x 8 tf32)
constexpr int kTgBStep = kTgN * 8 * 4;    // bytes of one K-step of B
constexpr int kTgOffAhi = 0;
constexpr int kTgOffAlo = kTgOffAhi + kTgSteps * kTgAStep;
constexpr int kTgOffBhi = kTgOffAlo + kTgSteps * kTgAStep;
constexpr int kTgOffBlo = kTgOffBhi + kTgSteps * kTgBStep;
constexpr int kTgSmem = kTgOffBlo + kTgSteps * kTgBStep;   // 64 KB
constexpr int kTgCols = kTgN;             // tensor-memory columns per CTA
// instruction descriptor: D f32, A/B tf32, both K-major, N = 128, M = 128
constexpr uint32_t kTgIdesc =
    (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTgN >> 3) << 17) | ((uint32_t)(kTgM >> 4) << 24);
static_assert(3 * (kTgSmem + 1024) <= 233472, "three CTAs per SM");
static_assert(3 * kTgCols <= 512, "tensor memory of three CTAs");

struct TgArgs {
  const float* L; long long strideL; int ldl;      // L^-1 (real, column-major)
  const float2* B; long long strideB; int ldb;     // complex, column-major
  int opB;                                          // 0: op(B)[k][j] = B[k][j]; 1: conj(B[j][k])
  float2* C; long long strideC; int ldc;
  const int* n;                                     // per-matrix size
  int lowerOnly;                                    // 1: only tiles holding an element with j <= i
  int* status;                                      // per-matrix status words
};

__global__ void __launch_bounds__(kTgThreads, 3) gemm_tc_kernel(TgArgs a) {
  extern __shared__ __align__(1024) unsigned char tg_sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmemSlot;
  __shared__ int sOk;
  const int b = blockIdx.z;
  const int n = a.n[b];
  const int i0 = blockIdx.x * kTgM, j0 = blockIdx.y * kTgNC;
  if (i0 >= n || j0 >= n) return;
  if (a.lowerOnly && j0 > i0 + kTgM - 1) return;
  const int kmax = min(n, i0 + kTgM);   // L^-1[i][k] = 0 for k > i
  const float* Lb = a.L + (long long)b * a.strideL;
  const float2* Bb = a.B + (long long)b * a.strideB;
  float2* Cb = a.C + (long long)b * a.strideC;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(tg_sm);
  const uint32_t bar = smem_u32(&mbar);
  if (tid == 0) {
    mbar_init(bar, 1);
    sOk = 1;
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemSlot)),
                 "r"(kTgCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmemSlot;
  uint32_t parity = 0;
  bool pending = false;
  const int row = i0 + tid;   // row of A staged by this thread
  // raw operands of one phase, loaded into registers one phase ahead: A row `row`, 32 k;
  // B units (complex column j, k quad) u = tid + 128 m
  float ra[kTgKP];
  float2 rb[4][4];
  auto load_phase = [&](int k0) {
#pragma unroll
    for (int kk = 0; kk < kTgKP; ++kk) {
      const int k = k0 + kk;
      ra[kk] = (row < n && k < n) ? Lb[row + (long long)k * a.ldl] : 0.f;
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int u = tid + kTgThreads * m;
      const int col = j0 + u % kTgNC, q = u / kTgNC;
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int k = k0 + 4 * q + e;
        float2 v = make_float2(0.f, 0.f);
        if (col < n && k < n) {
          if (a.opB == 0) {
            v = Bb[k + (long long)col * a.ldb];
          } else {
            v = Bb[col + (long long)k * a.ldb];
            v.y = -v.y;
          }
        }
        rb[m][e] = v;
      }
    }
  };
  load_phase(0);
  for (int k0 = 0; k0 < kmax; k0 += kTgKP) {
    // the operands of the previous phase must have been consumed
    if (tid == 0 && pending) {
      if (mbar_wait(bar, parity)) {
        parity ^= 1u;
        pending = false;
      } else {
        sOk = 0;
      }
    }
    __syncthreads();
    if (!sOk) break;
    // A: thread = row; 8 quads of k, each one 16-byte row chunk of a K-half
#pragma unroll
    for (int q = 0; q < kTgKP / 4; ++q) {
      float h[4], l[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) split_tf32(ra[4 * q + e], h[e], l[e]);
      const uint32_t off = (q >> 1) * kTgAStep + (q & 1) * (kTgAStep / 2) + tid * 16;
      st_shared_v4(sbase + kTgOffAhi + off, h[0], h[1], h[2], h[3]);
      st_shared_v4(sbase + kTgOffAlo + off, l[0], l[1], l[2], l[3]);
    }
    // B: real rows 2j (re), 2j+1 (im)
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int u = tid + kTgThreads * m;
      const int j = u % kTgNC, q = u / kTgNC;
      float rh[4], rl[4], ih[4], il[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        split_tf32(rb[m][e].x, rh[e], rl[e]);
        split_tf32(rb[m][e].y, ih[e], il[e]);
      }
      const uint32_t off = (q >> 1) * kTgBStep + (q & 1) * (kTgBStep / 2) + (2 * j) * 16;
      st_shared_v4(sbase + kTgOffBhi + off, rh[0], rh[1], rh[2], rh[3]);
      st_shared_v4(sbase + kTgOffBlo + off, rl[0], rl[1], rl[2], rl[3]);
      st_shared_v4(sbase + kTgOffBhi + off + 16, ih[0], ih[1], ih[2], ih[3]);
      st_shared_v4(sbase + kTgOffBlo + off + 16, il[0], il[1], il[2], il[3]);
    }
    // the next phase's operands are read from memory while this phase's MMAs run
    if (k0 + kTgKP < kmax) load_phase(k0 + kTgKP);
    // make the operand writes visible to the tensor core, then one thread issues
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int s = 0; s < kTgSteps; ++s) {
        const uint64_t dAh = tc_desc(sbase + kTgOffAhi + s * kTgAStep, kTgAStep / 2, 128);
        const uint64_t dAl = tc_desc(sbase + kTgOffAlo + s * kTgAStep, kTgAStep / 2, 128);
        const uint64_t dBh = tc_desc(sbase + kTgOffBhi + s * kTgBStep, kTgBStep / 2, 128);
        const uint64_t dBl = tc_desc(sbase + kTgOffBlo + s * kTgBStep, kTgBStep / 2, 128);
        tc_mma(tmem, dAh, dBh, kTgIdesc, (k0 > 0 || s > 0) ? 1u : 0u);
        tc_mma(tmem, dAh, dBl, kTgIdesc, 1u);
        tc_mma(tmem, dAl, dBh, kTgIdesc, 1u);
      }
      tc_commit(bar);
      pending = true;
    }
  }
  // accumulator complete
  if (tid == 0 && pending) {
    if (mbar_wait(bar, parity)) {
      parity ^= 1u;
      pending = false;
    } else {
      sOk = 0;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (sOk) {
    // warp w holds rows 32 w .. 32 w + 31 of the accumulator (one row per lane)
    const int i = i0 + warp * 32 + lane;
    const uint32_t tw = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c16 = 0; c16 < kTgN / 16; ++c16) {
      float r[16];
      tmem_ld16(tw + (uint32_t)(c16 * 16), r);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int col = j0 + c16 * 8 + c;
        if (i < n && col < n) Cb[i + (long long)col * a.ldc] = make_float2(r[2 * c], r[2 * c + 1]);
      }
    }
  }
  // after a timeout: wait once more (bounded) for MMAs still in flight, then release
  if (tid == 0) {
    if (pending) mbar_wait(bar, parity);
    if (!sOk) atomicOr(a.status + b, (int)kStatusTensorTimeout);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTgCols) : "memory");
  }
}

}  // namespace bippb200
