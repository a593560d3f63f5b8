// Virtual visibilities VV_l = X diag(s) X^H of every (time step, energy level) of a batch
// on the 5th-generation tensor cores (sm_100a, tcgen05), the contraction of
// src/host/virtual_vis.cpp:52-68 (V_k diag(scale d_k) V_k^H with the level's eigenvalues),
// plus an FP64 form for precision studies.
//
// X (the eigenvectors of a step, column-major, ld Nmax) is complex FP32; the columns of a
// level are the contiguous index range [kbeg, kend) (eigenvalues ascending) and s_k =
// kscale[k] = filter(d_k) / nVis. With A = X diag(s) and B = X,
//   Re C = A_re B_re^T + A_im B_im^T,   Im C = A_im B_re^T - A_re B_im^T,
// i.e. one real GEMM over K' = 2k: A' = [A_re | A_im] and, per complex output column j, the
// two real rows [B_re | B_im] (real part) and [-B_im | B_re] (imaginary part). A CTA tile
// is 128 rows x 64 complex columns (MMA M = 128, N = 128 real columns, FP32 accumulator in
// tensor memory); only tiles and entries of the lower triangle (i >= j) are formed, as the
// NUFFT reads VV_rs for r >= s. FP32 accuracy from split operands:
//   kind::tf32, 3xTF32:  a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi (hi = 11 significant bits)
//   kind::f16,  BF16x3:  a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi (hi = bf16(a), lo =
//                        bf16(a - hi): 16 significant bits in two bf16 values)
// Persistent CTAs walk the (step, level, tile) items; a level with no eigenvalue gives a
// zero tile (the reference returns VV = 0, src/host/virtual_vis.cpp:35-43). Every wait on
// the MMA completion barrier is bounded; a timeout sets the step's status bit and the CTA
// stops, freeing its tensor memory.
#pragma once

#include <cuda_bf16.h>

#include "common.cuh"
#include "tc_common.cuh"

namespace bippb200 {

constexpr int kVvThreads = 128;
constexpr int kVvM = 128;          // rows of VV per tile
constexpr int kVvNC = 64;          // complex columns of VV per tile
constexpr int kVvKC = 16;          // complex k per phase (K' = 32 real)
constexpr int kVvStep = 128 * 32;  // bytes of one MMA K-step of a 128-row operand (32 B of K per row)
constexpr int kVvCols = 128;       // tensor-memory columns per CTA (128 x 128 FP32)

// mode: 1 = 3xTF32, 2 = BF16x3 (operand bytes per row per phase: 128 / 64)
template <int MODE> struct VvShape {
  static constexpr int Steps = MODE == 1 ? 4 : 2;          // MMA K-steps per phase
  static constexpr int Operand = Steps * kVvStep;           // bytes of one operand (A or B, hi or lo)
  static constexpr int OffAhi = 0, OffAlo = Operand, OffBhi = 2 * Operand, OffBlo = 3 * Operand;
  // both modes request 64 KB, so that at most three CTAs (3 x 128 tensor-memory columns)
  // are resident on an SM and none waits in tcgen05.alloc behind a persistent CTA
  static constexpr int Smem = 4 * 4 * kVvStep;
  // instruction descriptor: D f32; A/B tf32 (2) or bf16 (1); both K-major; N = 128, M = 128
  static constexpr uint32_t Idesc = (1u << 4) | ((MODE == 1 ? 2u : 1u) << 7) | ((MODE == 1 ? 2u : 1u) << 10) |
                                    ((uint32_t)(128 >> 3) << 17) | ((uint32_t)(kVvM >> 4) << 24);
};
static_assert(3 * (VvShape<1>::Smem + 1024) <= 233472, "three CTAs per SM");

struct VvArgs {
  const float2* X; long long strideX; int ldx;   // eigenvectors per step
  const float* kscale; long long strideK;        // per-step column scales
  const int* kbeg; const int* kend;              // [step][level] column range
  const int* n;                                  // per-step matrix size
  float2* VV; long long strideStep, strideLevel; int ldv;
  int nSteps, nLevels, tilesI, tilesJ;
  int* status;                                   // per-step status words
};

__device__ __forceinline__ void mma_issue(uint32_t tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc,
                                          bool bf16) {
  if (bf16)
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
  else
    tc_mma(tmem, a, b, idesc, acc);
}

// bf16 split of two values packed as one 32-bit word each (low half = first value)
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat16 ah = __float2bfloat16_rn(a), bh = __float2bfloat16_rn(b);
  const __nv_bfloat16 al = __float2bfloat16_rn(a - __bfloat162float(ah));
  const __nv_bfloat16 bl = __float2bfloat16_rn(b - __bfloat162float(bh));
  hi = (uint32_t)__bfloat16_as_ushort(ah) | ((uint32_t)__bfloat16_as_ushort(bh) << 16);
  lo = (uint32_t)__bfloat16_as_ushort(al) | ((uint32_t)__bfloat16_as_ushort(bl) << 16);
}

__device__ __forceinline__ void st_shared_v4u(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}
__device__ __forceinline__ void st_shared_v2u(uint32_t addr, uint32_t a, uint32_t b) {
  asm volatile("st.shared.v2.b32 [%0], {%1, %2};" ::"r"(addr), "r"(a), "r"(b) : "memory");
}

// byte offset of 16-byte chunk c (K order within a phase) of operand row r
__device__ __forceinline__ uint32_t vv_chunk(int c, int r) {
  return (uint32_t)((c >> 1) * kVvStep + (c & 1) * (kVvStep / 2) + r * 16);
}

template <int MODE>
__global__ void __launch_bounds__(kVvThreads, 3) vv_tc_kernel(VvArgs a) {
  using S = VvShape<MODE>;
  constexpr bool kBf16 = MODE == 2;
  extern __shared__ __align__(1024) unsigned char vv_sm[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmemSlot;
  __shared__ int sOk;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t sbase = smem_u32(vv_sm);
  const uint32_t bar = smem_u32(&mbar);
  if (tid == 0) {
    mbar_init(bar, 1);
    sOk = 1;
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemSlot)),
                 "r"(kVvCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmemSlot;
  uint32_t parity = 0;
  bool pending = false;
  int lastStep = -1;
  const long long tilesPer = (long long)a.tilesI * a.tilesJ;
  const long long nItems = (long long)a.nSteps * a.nLevels * tilesPer;
  for (long long item = blockIdx.x; item < nItems; item += gridDim.x) {
    const int b = (int)(item / (tilesPer * a.nLevels));
    const long long rem = item % (tilesPer * a.nLevels);
    const int lvl = (int)(rem / tilesPer);
    const int t = (int)(rem % tilesPer);
    const int i0 = (t / a.tilesJ) * kVvM, j0 = (t % a.tilesJ) * kVvNC;
    const int n = a.n[b];
    if (i0 >= n || j0 >= n || j0 > i0 + kVvM - 1) continue;   // uniform across the CTA
    lastStep = b;
    const int z = b * a.nLevels + lvl;
    const int kb = a.kbeg[z], ke = a.kend[z];
    float2* C = a.VV + (long long)b * a.strideStep + (long long)lvl * a.strideLevel;
    if (kb >= ke) {
      // no eigenvalue in this level: a zero tile (lower entries)
      for (int e = tid; e < kVvM * kVvNC; e += kVvThreads) {
        const int i = i0 + e % kVvM, j = j0 + e / kVvM;
        if (i < n && j < n && i >= j) C[i + (long long)j * a.ldv] = make_float2(0.f, 0.f);
      }
      continue;
    }
    const float2* X = a.X + (long long)b * a.strideX;
    const float* ks = a.kscale + (long long)b * a.strideK;
    const int row = i0 + tid;
    // raw operands of one phase in registers, loaded one phase ahead: A row `row` (16
    // complex k); B units u = tid + 128 m: complex column j = u % 64, k quad q = u / 64
    float2 ra[kVvKC];
    float2 rb[2][4];
    auto load_phase = [&](int k0) {
#pragma unroll
      for (int kk = 0; kk < kVvKC; ++kk) {
        const int k = k0 + kk;
        float2 v = make_float2(0.f, 0.f);
        if (row < n && k < ke) {
          v = X[row + (long long)k * a.ldx];
          const float s = ks[k];
          v.x *= s;
          v.y *= s;
        }
        ra[kk] = v;
      }
#pragma unroll
      for (int m = 0; m < 2; ++m) {
        const int u = tid + kVvThreads * m;
        const int col = j0 + u % kVvNC, q = u / kVvNC;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int k = k0 + 4 * q + e;
          rb[m][e] = (col < n && k < ke) ? X[col + (long long)k * a.ldx] : make_float2(0.f, 0.f);
        }
      }
    };
    load_phase(kb);
    for (int k0 = kb; k0 < ke; k0 += kVvKC) {
      // the operands of the previous phase (or the previous tile) must have been consumed
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
      if (!kBf16) {
        // A: chunks 0..3 real parts (k quads), 4..7 imaginary parts
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float rh[4], rl[4], ih[4], il[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            split_tf32(ra[4 * q + e].x, rh[e], rl[e]);
            split_tf32(ra[4 * q + e].y, ih[e], il[e]);
          }
          st_shared_v4(sbase + S::OffAhi + vv_chunk(q, tid), rh[0], rh[1], rh[2], rh[3]);
          st_shared_v4(sbase + S::OffAlo + vv_chunk(q, tid), rl[0], rl[1], rl[2], rl[3]);
          st_shared_v4(sbase + S::OffAhi + vv_chunk(4 + q, tid), ih[0], ih[1], ih[2], ih[3]);
          st_shared_v4(sbase + S::OffAlo + vv_chunk(4 + q, tid), il[0], il[1], il[2], il[3]);
        }
        // B: row 2j = [B_re | B_im], row 2j + 1 = [-B_im | B_re]
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          const int u = tid + kVvThreads * m;
          const int j = u % kVvNC, q = u / kVvNC;
          float rh[4], rl[4], ih[4], il[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            split_tf32(rb[m][e].x, rh[e], rl[e]);
            split_tf32(rb[m][e].y, ih[e], il[e]);
          }
          st_shared_v4(sbase + S::OffBhi + vv_chunk(q, 2 * j), rh[0], rh[1], rh[2], rh[3]);
          st_shared_v4(sbase + S::OffBlo + vv_chunk(q, 2 * j), rl[0], rl[1], rl[2], rl[3]);
          st_shared_v4(sbase + S::OffBhi + vv_chunk(4 + q, 2 * j), ih[0], ih[1], ih[2], ih[3]);
          st_shared_v4(sbase + S::OffBlo + vv_chunk(4 + q, 2 * j), il[0], il[1], il[2], il[3]);
          st_shared_v4(sbase + S::OffBhi + vv_chunk(q, 2 * j + 1), -ih[0], -ih[1], -ih[2], -ih[3]);
          st_shared_v4(sbase + S::OffBlo + vv_chunk(q, 2 * j + 1), -il[0], -il[1], -il[2], -il[3]);
          st_shared_v4(sbase + S::OffBhi + vv_chunk(4 + q, 2 * j + 1), rh[0], rh[1], rh[2], rh[3]);
          st_shared_v4(sbase + S::OffBlo + vv_chunk(4 + q, 2 * j + 1), rl[0], rl[1], rl[2], rl[3]);
        }
      } else {
        // A: chunk 0 = real parts of k 0..7, 1 = of k 8..15, 2 / 3 = imaginary parts
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const float2 p0 = ra[8 * h + 2 * e], p1 = ra[8 * h + 2 * e + 1];
            split_bf16x2(p0.x, p1.x, rh[e], rl[e]);
            split_bf16x2(p0.y, p1.y, ih[e], il[e]);
          }
          st_shared_v4u(sbase + S::OffAhi + vv_chunk(h, tid), rh[0], rh[1], rh[2], rh[3]);
          st_shared_v4u(sbase + S::OffAlo + vv_chunk(h, tid), rl[0], rl[1], rl[2], rl[3]);
          st_shared_v4u(sbase + S::OffAhi + vv_chunk(2 + h, tid), ih[0], ih[1], ih[2], ih[3]);
          st_shared_v4u(sbase + S::OffAlo + vv_chunk(2 + h, tid), il[0], il[1], il[2], il[3]);
        }
        // B: k quad q fills bytes 8 (q & 1) .. of chunk q >> 1 (real) and 2 + (q >> 1) (imaginary)
#pragma unroll
        for (int m = 0; m < 2; ++m) {
          const int u = tid + kVvThreads * m;
          const int j = u % kVvNC, q = u / kVvNC;
          uint32_t rh[2], rl[2], ih[2], il[2], nh[2], nl[2];
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const float2 p0 = rb[m][2 * e], p1 = rb[m][2 * e + 1];
            split_bf16x2(p0.x, p1.x, rh[e], rl[e]);
            split_bf16x2(p0.y, p1.y, ih[e], il[e]);
            split_bf16x2(-p0.y, -p1.y, nh[e], nl[e]);
          }
          const uint32_t byte = 8u * (uint32_t)(q & 1);
          const int cr = q >> 1, ci = 2 + (q >> 1);
          st_shared_v2u(sbase + S::OffBhi + vv_chunk(cr, 2 * j) + byte, rh[0], rh[1]);
          st_shared_v2u(sbase + S::OffBlo + vv_chunk(cr, 2 * j) + byte, rl[0], rl[1]);
          st_shared_v2u(sbase + S::OffBhi + vv_chunk(ci, 2 * j) + byte, ih[0], ih[1]);
          st_shared_v2u(sbase + S::OffBlo + vv_chunk(ci, 2 * j) + byte, il[0], il[1]);
          st_shared_v2u(sbase + S::OffBhi + vv_chunk(cr, 2 * j + 1) + byte, nh[0], nh[1]);
          st_shared_v2u(sbase + S::OffBlo + vv_chunk(cr, 2 * j + 1) + byte, nl[0], nl[1]);
          st_shared_v2u(sbase + S::OffBhi + vv_chunk(ci, 2 * j + 1) + byte, rh[0], rh[1]);
          st_shared_v2u(sbase + S::OffBlo + vv_chunk(ci, 2 * j + 1) + byte, rl[0], rl[1]);
        }
      }
      // the next phase's operands are read from memory while this phase's MMAs run
      if (k0 + kVvKC < ke) load_phase(k0 + kVvKC);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
#pragma unroll
        for (int s = 0; s < S::Steps; ++s) {
          const uint64_t dAh = tc_desc(sbase + S::OffAhi + s * kVvStep, kVvStep / 2, 128);
          const uint64_t dAl = tc_desc(sbase + S::OffAlo + s * kVvStep, kVvStep / 2, 128);
          const uint64_t dBh = tc_desc(sbase + S::OffBhi + s * kVvStep, kVvStep / 2, 128);
          const uint64_t dBl = tc_desc(sbase + S::OffBlo + s * kVvStep, kVvStep / 2, 128);
          mma_issue(tmem, dAh, dBh, S::Idesc, (k0 > kb || s > 0) ? 1u : 0u, kBf16);
          mma_issue(tmem, dAh, dBl, S::Idesc, 1u, kBf16);
          mma_issue(tmem, dAl, dBh, S::Idesc, 1u, kBf16);
        }
        tc_commit(bar);
        pending = true;
      }
    }
    // accumulator complete
    if (tid == 0 && pending && sOk) {
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
    if (!sOk) break;
    // warp w holds rows 32 w .. 32 w + 31 (one per lane); columns (2 j, 2 j + 1) = (re, im)
    const int i = i0 + warp * 32 + lane;
    const uint32_t tw = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int c16 = 0; c16 < 128 / 16; ++c16) {
      float r[16];
      tmem_ld16(tw + (uint32_t)(c16 * 16), r);
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const int j = j0 + c16 * 8 + c;
        if (i < n && j < n && i >= j) C[i + (long long)j * a.ldv] = make_float2(r[2 * c], r[2 * c + 1]);
      }
    }
    // the next tile's MMAs overwrite the accumulator only after every warp has read it
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
  }
  // after a timeout: wait once more (bounded) for MMAs still in flight, then release
  if (tid == 0) {
    if (pending) mbar_wait(bar, parity);
    if (!sOk && lastStep >= 0) atomicOr(a.status + lastStep, (int)kStatusTensorTimeout);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kVvCols) : "memory");
  }
}

// FP64 form (precision studies): the same products with FP64 arithmetic on the FP32
// eigenvectors and scales, rounded to complex FP32 at the end. 64 x 64 tiles, 256
// threads with 4 x 4 outputs each, k staged 16 at a time in shared memory.
constexpr int kVv64Tile = 64, kVv64K = 16, kVv64Threads = 256;

static __global__ void __launch_bounds__(kVv64Threads) vv_fp64_kernel(VvArgs a) {
  const int z = blockIdx.z;
  const int b = z / a.nLevels, lvl = z % a.nLevels;
  const int n = a.n[b];
  const int i0 = blockIdx.y * kVv64Tile, j0 = blockIdx.x * kVv64Tile;
  if (i0 >= n || j0 >= n || j0 > i0 + kVv64Tile - 1) return;
  const int kb = a.kbeg[z], ke = a.kend[z];
  const float2* X = a.X + (long long)b * a.strideX;
  const float* ks = a.kscale + (long long)b * a.strideK;
  float2* C = a.VV + (long long)b * a.strideStep + (long long)lvl * a.strideLevel;
  __shared__ double2 As[kVv64K][kVv64Tile + 1];
  __shared__ double2 Bs[kVv64K][kVv64Tile + 1];
  const int tid = threadIdx.x, tr = tid % 16, tc = tid / 16;
  double2 acc[4][4];
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[p][q] = make_double2(0.0, 0.0);
  for (int k0 = kb; k0 < ke; k0 += kVv64K) {
    for (int e = tid; e < kVv64K * kVv64Tile; e += kVv64Threads) {
      const int r = e % kVv64Tile, kk = e / kVv64Tile, k = k0 + kk;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (k < ke) {
        if (i0 + r < n) {
          const float2 x = X[i0 + r + (long long)k * a.ldx];
          const double s = (double)ks[k];
          va = make_double2((double)x.x * s, (double)x.y * s);
        }
        if (j0 + r < n) {
          const float2 x = X[j0 + r + (long long)k * a.ldx];
          vb = make_double2((double)x.x, -(double)x.y);   // conj(B[j, k])
        }
      }
      As[kk][r] = va;
      Bs[kk][r] = vb;
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < kVv64K; ++kk) {
      double2 av[4], bv[4];
#pragma unroll
      for (int p = 0; p < 4; ++p) av[p] = As[kk][tr + 16 * p];
#pragma unroll
      for (int q = 0; q < 4; ++q) bv[q] = Bs[kk][tc + 16 * q];
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) cfma(acc[p][q], av[p], bv[q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + tr + 16 * p, j = j0 + tc + 16 * q;
      if (i < n && j < n && i >= j) C[i + (long long)j * a.ldv] = make_float2((float)acc[p][q].x, (float)acc[p][q].y);
    }
}

}  // namespace bippb200
