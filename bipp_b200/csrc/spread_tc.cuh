// NUFFT spreading on the 5th-generation tensor cores (sm_100a, tcgen05).
//
// For one output tile of 16 x 8 (x, y) cells and 8 w-planes, the spread grid is a sum of
// separable outer products over the points ("visits") that reach the tile:
//     G[(x,y), (w,c)] = sum_p  phi_x,p(x) phi_y,p(y)  *  phi_w,p(w) v_p,c
// i.e. the product of A (128 cells x K visits) and B (K visits x 16 CH columns: 8 planes x
// CH = 4 or 8 channels x re/im). Threads write A and B for 16 visits at a time into shared memory
// (canonical K-major, no swizzle), one thread issues tcgen05.mma (kind::tf32) into a
// 128 x 16 CH FP32 accumulator in tensor memory, and the epilogue reads it back with
// tcgen05.ld and writes the tile once. FP32 accuracy comes from the 3xTF32 split
// a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi (a_hi = tf32(a), a_lo = tf32(a - a_hi)).
// Every wait on the MMA completion barrier is bounded; a timeout sets an error flag
// that the host turns into an error, and the CTA still frees its tensor memory.
#pragma once

#include <cstdint>

#include <cuda_fp16.h>

#include "nufft_kernels.cuh"
#include "tc_common.cuh"

namespace bippb200 {

constexpr int kTcThreads = 128;
constexpr int kTcVisits = 16;                 // visits per phase
constexpr int kTcSteps = kTcVisits / 8;       // MMA K-steps per phase (K = 8 for tf32)
constexpr int kTcM = kTX * kTY;               // 128 accumulator rows (cells)
constexpr int kTcMaxChan = 8;                 // channels handled by the tensor-core kernel
// shared-memory layout (bytes); one K-step of A is 128 rows x 8 tf32
constexpr int kTcAStep = kTcM * 8 * 4;
// per-visit kernel values at every tile position (zero outside the support) and the
// channel values, stored position-major, 16 visits per row, so that the operand builders
// read 4 visits with one 16-byte load. Rows read by 8 different threads of a quarter warp
// (x positions, channel values) have their 16-byte chunks permuted by the row (tab_sw):
// conflict-free for those loads and for the writes of a thread per visit.
constexpr int kTcVS = kTcVisits;
__device__ __forceinline__ int tab_sw(int row, int v) {
  return row * kTcVS + ((((v >> 2) ^ (row >> 1)) & 3) << 2) + (v & 3);
}
static_assert(kTX == 16 && kTY == 8 && kTW == 8 && kTcVisits == 16, "prep mapping assumes 16 x 8 x 8 tiles, 16 visits");

// Shape of the kernel for CH channels (4 or 8), STAGES operand stages (1, or 2 so that a
// phase's operands are built while the previous phase's MMAs run) and the place of the A
// operand (AT: tensor memory, written by each thread into its own lane with tcgen05.st;
// otherwise shared memory): accumulator 128 x N, N = 8 planes x CH channels x re/im; one
// K-step of B is N rows x 8 tf32; CTAs per SM bounded by TMEM (512 columns) and shared
// memory. With A in tensor memory the tensor cores read only B from shared memory, and
// the threads store only B there: about half of the shared-memory traffic of a phase.
// F16: operands split into FP16 hi + lo (kind::f16, K = 16: one K-step per 16-point
// phase; half the operand bytes and MMAs of the tf32 split, so that two stages fit the
// shared memory of 8 CTAs per SM). B is built from values scaled per channel into
// [-1, 1] (FP16 range), the epilogue scales back.
constexpr int tc_pow2_cols(int c) { return c <= 32 ? 32 : c <= 64 ? 64 : c <= 128 ? 128 : c <= 256 ? 256 : 512; }
template <int CH, int STAGES = 1, bool AT = false, bool F16 = false>
struct TcShape {
  static constexpr int N = kTW * 2 * CH;
  static constexpr int KSteps = F16 ? 1 : kTcSteps;              // MMA K-steps per phase
  static constexpr int AStageCols = AT ? 2 * kTcSteps * 8 : 0;   // A_hi, A_lo of a phase (K = 16 each)
  static constexpr int AColBase = N;                             // A of stage s at AColBase + s AStageCols
  static constexpr int Cols = tc_pow2_cols(N + STAGES * AStageCols);   // tensor-memory columns per CTA
  static constexpr int BStep = N * 8 * 4;
  static constexpr int OffAhi = 0;                // operands of stage 0; stage s at + s StageBytes
  static constexpr int OffAlo = OffAhi + (AT ? 0 : KSteps * kTcAStep);
  static constexpr int OffBhi = OffAlo + (AT ? 0 : KSteps * kTcAStep);
  static constexpr int OffBlo = OffBhi + KSteps * BStep;
  static constexpr int StageBytes = OffBlo + KSteps * BStep;
  static constexpr int OffEx = STAGES * StageBytes;        // float [16 x][kTcVS]
  static constexpr int OffEy = OffEx + kTX * kTcVS * 4;    // float [8 y][kTcVS]
  static constexpr int OffEw = OffEy + kTY * kTcVS * 4;    // float [8 w][kTcVS]
  static constexpr int OffVal = OffEw + kTW * kTcVS * 4;   // float [2 CH (channel, re/im)][kTcVS]
  static constexpr int Smem = OffVal + 2 * CH * kTcVS * 4;
  static constexpr int BySmem = 233472 / (Smem + 512 + 1024);
  static constexpr int MinBlocks = (512 / Cols) < BySmem ? (512 / Cols) : BySmem;   // CTAs per SM
  // instruction descriptor: D f32, A/B tf32 (2) or f16 (0), both K-major, N, M = 128
  static constexpr uint32_t Idesc = (1u << 4) | ((F16 ? 0u : 2u) << 7) | ((F16 ? 0u : 2u) << 10) |
                                    ((uint32_t)(N >> 3) << 17) | ((uint32_t)(kTcM >> 4) << 24);
  static_assert(CH == 4 || CH == 8, "4 or 8 channels");
  static_assert(!(AT && F16), "tensor-memory A with the tf32 split only");
  static_assert(N % 16 == 0 && N <= 256, "MMA N for M = 128");
  static_assert(OffEx % 1024 == 0, "operand blocks 1 KB aligned");
  static_assert(STAGES == 1 || STAGES == 2, "one or two operand stages");
  static_assert(MinBlocks >= 1 && MinBlocks * (Smem + 512 + 1024) <= 233472,
                "shared memory (dynamic + static <= 512 B + 1 KB reserved) for MinBlocks CTAs per SM");
};

// FP16 hi + lo of two values, each pair packed in one 32-bit word (low half = first):
// hi rounded to FP16, lo = FP16 of the exact FP32 remainder
__device__ __forceinline__ void split_f16x2(float2 x, uint32_t& hi, uint32_t& lo) {
  const __half2 h = __float22half2_rn(x);
  const float2 hf = __half22float2(h);
  const __half2 l = __float22half2_rn(make_float2(x.x - hf.x, x.y - hf.y));
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

__device__ __forceinline__ void tc_mma_f16(uint32_t tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void st_shared_v4w(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

// The 27 (source direction d, crossing bits) pairs whose key ranges reach a tile, in
// the order tile_ranges() visits them: d in 0..7, bits a superset of d.
__device__ __forceinline__ int tc_range_pair(int j) {
  int n = 0;
  for (int d = 0; d < 8; ++d)
    for (int bits = 0; bits < 8; ++bits)
      if ((bits & d) == d) {
        if (n == j) return d | (bits << 3);
        ++n;
      }
  return -1;
}

// Persistent: each CTA takes work items blockIdx.x, blockIdx.x + gridDim.x, ... or, with
// a work counter, the next item of the (load-ordered) list whenever it is free
template <int CH, int STAGES, bool AT = false, bool F16 = false>
static __global__ void __launch_bounds__(kTcThreads, TcShape<CH, STAGES, AT, F16>::MinBlocks)
spread_tc_kernel(NufftGeom g, const int* __restrict__ offsets, const PtRec* __restrict__ rec,
                 const float2* __restrict__ vals, long long valStride, int nch, const SpreadItem* __restrict__ items,
                 int nItems, int tw0, int slabPlanes, float2* __restrict__ grid, int* __restrict__ errFlag,
                 int* __restrict__ workCounter, const unsigned* __restrict__ valScale = nullptr) {
  using S = TcShape<CH, STAGES, AT, F16>;
  extern __shared__ __align__(128) unsigned char sm[];
  __shared__ __align__(8) uint64_t mbar[STAGES];   // MMA completion of the phases of each stage
  __shared__ uint32_t tmemSlot;
  __shared__ int rBeg[27], rPre[28];
  __shared__ int sOk, sItem;
  const int tid = threadIdx.x, warp = tid >> 5;
  const uint32_t sbase = smem_u32(sm);
  float* ex = reinterpret_cast<float*>(sm + S::OffEx);
  float* ey = reinterpret_cast<float*>(sm + S::OffEy);
  float* ew = reinterpret_cast<float*>(sm + S::OffEw);
  float* val = reinterpret_cast<float*>(sm + S::OffVal);
  if (tid == 0) {
    for (int st = 0; st < STAGES; ++st) mbar_init(smem_u32(&mbar[st]), 1);
    sOk = 1;
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmemSlot)),
                 "r"(S::Cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmemSlot;
  const uint32_t tmemWarp = tmem + ((uint32_t)(warp * 32) << 16);
  const float invHalf = 2.0f / (float)g.W;
  const int W = g.W;
  const int xm = tid % kTX, ym = tid / kTX;   // cell of accumulator row tid
  const int lane = tid & 31;
  const int myPair = (lane < 27) ? tc_range_pair(lane) : -1;
  // thread 0's view of each stage's barrier: its phase parity and whether a commit of
  // that stage has not been waited for
  // (bit st of each word), kept in registers
  uint32_t parityBits = 0, pendingBits = 0;
  // bounded wait (thread 0) for stage st's last commit; false on timeout
  auto wait_stage = [&](int st) {
    if (!((pendingBits >> st) & 1u)) return true;
    if (!mbar_wait(smem_u32(&mbar[st]), (parityBits >> st) & 1u)) return false;
    parityBits ^= 1u << st;
    pendingBits &= ~(1u << st);
    return true;
  };
  for (int item = blockIdx.x;; item += gridDim.x) {
    if (workCounter) {
      // every thread has read the previous sItem (the item ends with a barrier)
      if (tid == 0) sItem = atomicAdd(workCounter, 1);
      __syncthreads();
      item = sItem;
    }
    if (item >= nItems) break;
    const SpreadItem it = items[item];
    const int tx = it.tile % g.ntx, ty = (it.tile / g.ntx) % g.nty, tw = it.tile / (g.ntx * g.nty);
    const int x0 = tx * kTX, y0 = ty * kTY, w0 = tw * kTW;
    if (warp == 0) {
      // lane j < 27: key range of pair j (empty when the source tile lies below w = 0)
      int beg = 0, len = 0;
      if (myPair >= 0) {
        const int d = myPair & 7, bits = myPair >> 3;
        const int stw = tw - ((d >> 2) & 1);
        if (stw >= 0) {
          const int stx = (tx - (d & 1) + g.ntx) % g.ntx;
          const int sty = (ty - ((d >> 1) & 1) + g.nty) % g.nty;
          const int key = ((stw * g.nty + sty) * g.ntx + stx) * 8 + bits;
          beg = offsets[key];
          len = offsets[key + 1] - beg;
        }
      }
      int incl = len;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      if (lane < 27) {
        rBeg[lane] = beg;
        rPre[lane] = incl - len;
      }
      if (lane == 26) rPre[27] = incl;
    }
    __syncthreads();
    const int lo = (int)((long long)it.load * it.part / it.nparts);
    const int hi = (int)((long long)it.load * (it.part + 1) / it.nparts);
    const int nvis = hi - lo;
    // thread (visit v, role a): a = 0..3: x positions 4a..4a+3, a = 4, 5: y positions,
    // a = 6, 7: w planes 4(a-6)..+3 and channels CH/2 (a-6) .. CH/2 (a-5) - 1. The point
    // data of the next phase are loaded into registers while the current phase is built.
    constexpr int CPR = CH / 2;   // channels per value role
    const int pv = tid & 15, pa = tid >> 4;
    // F16: this thread's value channels scaled into [-1, 1] (valScale: per-channel max of
    // |Re|, |Im| as FP32 bits)
    float invS[CPR];
#pragma unroll
    for (int cc = 0; cc < CPR; ++cc) {
      invS[cc] = 1.f;
      if constexpr (F16) {
        const int c = CPR * (pa >= 6 ? pa - 6 : 0) + cc;
        const float sc = (c < nch) ? __uint_as_float(valScale[c]) : 0.f;
        invS[cc] = sc > 0.f ? 1.f / sc : 0.f;
      }
    }
    int ri = 0;
    int pfL = 0;
    float pfD = 0.f;
    float2 pfX[CPR];
#pragma unroll
    for (int c = 0; c < CPR; ++c) pfX[c] = make_float2(0.f, 0.f);
    auto fetch = [&](int vb) {
      if (pv < min(kTcVisits, nvis - vb)) {
        const int q = lo + vb + pv;
        while (q >= rPre[ri + 1]) ++ri;
        const int p = rBeg[ri] + (q - rPre[ri]);
        const PtRec* pr = rec + p;
        if (pa < 4) {
          pfL = __ldg(&pr->ix0);
          pfD = __ldg(&pr->dx);
        } else if (pa < 6) {
          pfL = __ldg(&pr->iy0);
          pfD = __ldg(&pr->dy);
        } else {
          pfL = __ldg(&pr->iw0);
          pfD = __ldg(&pr->dw);
          // values of a point are contiguous ([point][channel])
#pragma unroll
          for (int cc = 0; cc < CPR; ++cc) {
            const int c = CPR * (pa - 6) + cc;
            pfX[cc] = (c < nch) ? vals[(long long)p * nch + c] : make_float2(0.f, 0.f);
          }
        }
      }
    };
    fetch(0);
    for (int v0 = 0; v0 < nvis; v0 += kTcVisits) {
      const int nk = min(kTcVisits, nvis - v0);
      const int steps = F16 ? 1 : (nk + 7) >> 3;
      const int kpad = F16 ? kTcVisits : steps * 8;   // visits of the phase's K-steps
      // operand stage of this phase
      const int stg = STAGES == 1 ? 0 : (v0 / kTcVisits) & 1;
      const uint32_t sstage = sbase + (uint32_t)(stg * S::StageBytes);
      // per-visit tables from the prefetched point data (the tensor cores read only the
      // operand blocks, so the tables are rebuilt while the previous phase's MMAs run)
      {
        float* tab = (pa < 4) ? ex : (pa < 6) ? ey : ew;
        const bool swz = pa < 4;
        const int first = 4 * ((pa < 4) ? pa : (pa < 6) ? pa - 4 : pa - 6);   // first table row of this role
        if (pv < nk) {
          int l = pfL;
          // periodic offset of the support start from the tile, in (-n/2, n/2]: the start
          // lies in [-n/2 - W/2, n/2) and the tile origin in [0, n), so the difference
          // lies in (-3n/2 - W/2, n/2) and two conditional additions wrap it
          if (pa < 6) {
            const int np = (pa < 4) ? g.nx : g.ny;
            l -= (pa < 4) ? x0 : y0;
            if (l <= -(np >> 1)) l += np;
            if (l <= -(np >> 1)) l += np;
            if (l > (np >> 1)) l -= np;
          } else {
            l -= w0;
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int j = first + i - l;   // support index of tile position first + i
            tab[swz ? tab_sw(first + i, pv) : (first + i) * kTcVS + pv] =
                ((unsigned)j < (unsigned)W) ? es_kernel(((float)j - pfD) * invHalf, g.beta) : 0.f;
          }
          if (pa >= 6) {
#pragma unroll
            for (int cc = 0; cc < CPR; ++cc) {
              const int c = CPR * (pa - 6) + cc;
              val[tab_sw(2 * c, pv)] = pfX[cc].x * invS[cc];
              val[tab_sw(2 * c + 1, pv)] = pfX[cc].y * invS[cc];
            }
          }
        } else if (pv < kpad) {
          // padding visits of the last K-step contribute nothing (values too: 0 x stale
          // shared memory could be 0 x NaN)
#pragma unroll
          for (int i = 0; i < 4; ++i) tab[swz ? tab_sw(first + i, pv) : (first + i) * kTcVS + pv] = 0.f;
          if (pa >= 6)
            for (int c = 2 * CPR * (pa - 6); c < 2 * CPR * (pa - 5); ++c) val[tab_sw(c, pv)] = 0.f;
        }
      }
      // the operands of this stage's previous phase must have been consumed before they
      // are rewritten (with two stages, the MMAs of the phase before run meanwhile)
      if (tid == 0 && !wait_stage(stg)) sOk = 0;
      if constexpr (AT) tc_fence_before();
      __syncthreads();
      if constexpr (AT) tc_fence_after();   // the stage's tensor memory is free to rewrite
      if (!sOk) break;
      if (v0 + kTcVisits < nvis) fetch(v0 + kTcVisits);
      // A: row tid (cell xm, ym), 8 visits per K-step
      if constexpr (F16) {
        // one K-step of 16 visits: FP16 hi/lo, k 0-7 and 8-15 in the two 16-byte halves
        uint32_t h[8], l[8];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const float4 xq = *reinterpret_cast<const float4*>(ex + tab_sw(xm, 4 * q));
          const float4 yq = *reinterpret_cast<const float4*>(ey + ym * kTcVS + 4 * q);
          split_f16x2(__fmul2_rn(make_float2(xq.x, xq.y), make_float2(yq.x, yq.y)), h[2 * q], l[2 * q]);
          split_f16x2(__fmul2_rn(make_float2(xq.z, xq.w), make_float2(yq.z, yq.w)), h[2 * q + 1], l[2 * q + 1]);
        }
        const uint32_t ah = sstage + S::OffAhi + tid * 16, al = sstage + S::OffAlo + tid * 16;
        st_shared_v4w(ah, h[0], h[1], h[2], h[3]);
        st_shared_v4w(ah + kTcAStep / 2, h[4], h[5], h[6], h[7]);
        st_shared_v4w(al, l[0], l[1], l[2], l[3]);
        st_shared_v4w(al + kTcAStep / 2, l[4], l[5], l[6], l[7]);
      }
      for (int s = 0; s < (F16 ? 0 : steps); ++s) {
        float h[8], l[8];
        {
          const float4 x0 = *reinterpret_cast<const float4*>(ex + tab_sw(xm, 8 * s));
          const float4 x1 = *reinterpret_cast<const float4*>(ex + tab_sw(xm, 8 * s + 4));
          const float4 y0 = *reinterpret_cast<const float4*>(ey + ym * kTcVS + 8 * s);
          const float4 y1 = *reinterpret_cast<const float4*>(ey + ym * kTcVS + 8 * s + 4);
          // products and splits two at a time (packed FP32x2)
          const float2 pr[4] = {__fmul2_rn(make_float2(x0.x, x0.y), make_float2(y0.x, y0.y)),
                                __fmul2_rn(make_float2(x0.z, x0.w), make_float2(y0.z, y0.w)),
                                __fmul2_rn(make_float2(x1.x, x1.y), make_float2(y1.x, y1.y)),
                                __fmul2_rn(make_float2(x1.z, x1.w), make_float2(y1.z, y1.w))};
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            float2 hi2, lo2;
            split_tf32x2(pr[t], hi2, lo2);
            h[2 * t] = hi2.x; h[2 * t + 1] = hi2.y;
            l[2 * t] = lo2.x; l[2 * t + 1] = lo2.y;
          }
        }
        if constexpr (AT) {
          // K-step s of A_hi at column +8 s, of A_lo at +16 + 8 s (row tid = lane tid)
          const uint32_t ta = tmemWarp + (uint32_t)(S::AColBase + stg * S::AStageCols + 8 * s);
          tmem_st8(ta, h);
          tmem_st8(ta + 16, l);
        } else {
          const uint32_t ah = sstage + S::OffAhi + s * kTcAStep + tid * 16;
          const uint32_t al = sstage + S::OffAlo + s * kTcAStep + tid * 16;
          st_shared_v4(ah, h[0], h[1], h[2], h[3]);
          st_shared_v4(ah + kTcAStep / 2, h[4], h[5], h[6], h[7]);
          st_shared_v4(al, l[0], l[1], l[2], l[3]);
          st_shared_v4(al + kTcAStep / 2, l[4], l[5], l[6], l[7]);
        }
      }
      // B: row n = plane * 2 CH + channel * 2 + (re|im); TPR threads per row, each with
      // VPT visits of the K-step
      if constexpr (F16) {
        // one K-step of 16 visits; TPR threads per row, each with 8 (TPR = 2) or 16 visits
        constexpr int TPR = kTcThreads / S::N, VPT = kTcVisits / TPR;
        const int n = tid % S::N, kh = tid / S::N;
        const int plane = n / (2 * CH), cc = n % (2 * CH);
#pragma unroll
        for (int q = 0; q < VPT / 8; ++q) {
          const int v = kh * VPT + 8 * q;   // first visit of this 16-byte chunk
          const float4 e0 = *reinterpret_cast<const float4*>(ew + plane * kTcVS + v);
          const float4 e1 = *reinterpret_cast<const float4*>(ew + plane * kTcVS + v + 4);
          const float4 c0 = *reinterpret_cast<const float4*>(val + tab_sw(cc, v));
          const float4 c1 = *reinterpret_cast<const float4*>(val + tab_sw(cc, v + 4));
          uint32_t h[4], l[4];
          split_f16x2(__fmul2_rn(make_float2(e0.x, e0.y), make_float2(c0.x, c0.y)), h[0], l[0]);
          split_f16x2(__fmul2_rn(make_float2(e0.z, e0.w), make_float2(c0.z, c0.w)), h[1], l[1]);
          split_f16x2(__fmul2_rn(make_float2(e1.x, e1.y), make_float2(c1.x, c1.y)), h[2], l[2]);
          split_f16x2(__fmul2_rn(make_float2(e1.z, e1.w), make_float2(c1.z, c1.w)), h[3], l[3]);
          const uint32_t off = (uint32_t)((v >> 3) * (S::BStep / 2) + n * 16);
          st_shared_v4w(sstage + S::OffBhi + off, h[0], h[1], h[2], h[3]);
          st_shared_v4w(sstage + S::OffBlo + off, l[0], l[1], l[2], l[3]);
        }
      } else {
        constexpr int TPR = kTcThreads / S::N, VPT = 8 / TPR;
        const int n = tid % S::N, kh = tid / S::N;
        const int plane = n / (2 * CH), cc = n % (2 * CH);
        for (int s = 0; s < steps; ++s) {
#pragma unroll
          for (int q = 0; q < VPT / 4; ++q) {
            const int k0 = kh * VPT + 4 * q;   // first visit of this 16-byte group
            float h[4], l[4];
            {
              const int v = s * 8 + k0;
              const float4 e4 = *reinterpret_cast<const float4*>(ew + plane * kTcVS + v);
              const float4 c4 = *reinterpret_cast<const float4*>(val + tab_sw(cc, v));
              const float2 p0 = __fmul2_rn(make_float2(e4.x, e4.y), make_float2(c4.x, c4.y));
              const float2 p1 = __fmul2_rn(make_float2(e4.z, e4.w), make_float2(c4.z, c4.w));
              float2 h0, l0, h1, l1;
              split_tf32x2(p0, h0, l0);
              split_tf32x2(p1, h1, l1);
              h[0] = h0.x; h[1] = h0.y; h[2] = h1.x; h[3] = h1.y;
              l[0] = l0.x; l[1] = l0.y; l[2] = l1.x; l[3] = l1.y;
            }
            const uint32_t bh = sstage + S::OffBhi + s * S::BStep + (k0 >> 2) * (S::BStep / 2) + n * 16;
            const uint32_t bl = sstage + S::OffBlo + s * S::BStep + (k0 >> 2) * (S::BStep / 2) + n * 16;
            st_shared_v4(bh, h[0], h[1], h[2], h[3]);
            st_shared_v4(bl, l[0], l[1], l[2], l[3]);
          }
        }
      }
      // make the operand writes visible to the tensor core, then one thread issues
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      if constexpr (AT) {
        tmem_st_wait();
        tc_fence_before();
      }
      __syncthreads();
      if (tid == 0) {
        tc_fence_after();
        for (int s = 0; s < steps; ++s) {
          const uint64_t dBh = tc_desc(sstage + S::OffBhi + s * S::BStep, S::BStep / 2, 128);
          const uint64_t dBl = tc_desc(sstage + S::OffBlo + s * S::BStep, S::BStep / 2, 128);
          if constexpr (F16) {
            const uint64_t dAh = tc_desc(sstage + S::OffAhi, kTcAStep / 2, 128);
            const uint64_t dAl = tc_desc(sstage + S::OffAlo, kTcAStep / 2, 128);
            tc_mma_f16(tmem, dAh, dBh, S::Idesc, v0 > 0 ? 1u : 0u);
            tc_mma_f16(tmem, dAh, dBl, S::Idesc, 1u);
            tc_mma_f16(tmem, dAl, dBh, S::Idesc, 1u);
          } else if constexpr (AT) {
            const uint32_t aHi = tmem + (uint32_t)(S::AColBase + stg * S::AStageCols + 8 * s);
            tc_mma_ta(tmem, aHi, dBh, S::Idesc, (v0 > 0 || s > 0) ? 1u : 0u);
            tc_mma_ta(tmem, aHi, dBl, S::Idesc, 1u);
            tc_mma_ta(tmem, aHi + 16, dBh, S::Idesc, 1u);
          } else {
            const uint64_t dAh = tc_desc(sstage + S::OffAhi + s * kTcAStep, kTcAStep / 2, 128);
            const uint64_t dAl = tc_desc(sstage + S::OffAlo + s * kTcAStep, kTcAStep / 2, 128);
            tc_mma(tmem, dAh, dBh, S::Idesc, (v0 > 0 || s > 0) ? 1u : 0u);
            tc_mma(tmem, dAh, dBl, S::Idesc, 1u);
            tc_mma(tmem, dAl, dBh, S::Idesc, 1u);
          }
        }
        tc_commit(smem_u32(&mbar[stg]));
        pendingBits |= 1u << stg;
      }
    }
    // accumulator complete (every stage's last commit waited for)
    if (tid == 0) {
#pragma unroll
      for (int st = 0; st < STAGES; ++st)
        if (sOk && !wait_stage(st)) sOk = 0;
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (!sOk) break;
    if (nvis > 0) {
      const int twl = tw - tw0;
      constexpr int PPB = 16 / (2 * CH);   // planes per 16-column block
#pragma unroll
      for (int q = 0; q < S::N / 16; ++q) {
        float r[16];
        tmem_ld16(tmemWarp + (uint32_t)(q * 16), r);
#pragma unroll
        for (int pl = 0; pl < PPB; ++pl) {
          const int plane = twl * kTW + q * PPB + pl;
#pragma unroll
          for (int c = 0; c < CH; ++c) {
            if (c < nch) {
              float2 v = make_float2(r[pl * 2 * CH + 2 * c], r[pl * 2 * CH + 2 * c + 1]);
              if constexpr (F16) {
                const float sc = __uint_as_float(__ldg(valScale + c));   // undo the value scaling
                v.x *= sc;
                v.y *= sc;
              }
              float2* dst = grid + slab_index(g, nch, slabPlanes, c, plane, y0 + ym, x0 + xm);
              if (it.nparts == 1) {
                *dst = v;
              } else {
                atomicAdd(&dst->x, v.x);
                atomicAdd(&dst->y, v.y);
              }
            }
          }
        }
      }
    }
    // tensor-memory reads done before the next tile's first MMA overwrites it
    tc_fence_before();
    __syncthreads();
  }
  // after a timeout: wait once more (bounded) for MMAs still in flight, then release
  if (tid == 0) {
#pragma unroll
    for (int st = 0; st < STAGES; ++st)
      if ((pendingBits >> st) & 1u) mbar_wait(smem_u32(&mbar[st]), (parityBits >> st) & 1u);
    if (!sOk) atomicOr(errFlag, 1);
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(S::Cols) : "memory");
  }
}

// Clear the listed tiles of one slab (empty tiles and tiles spread in several parts):
// one CTA per listed tile, thread = cell, a 128-byte row of the tile per warp store
static __global__ void __launch_bounds__(kTcThreads)
clear_tiles_kernel(NufftGeom g, const int* __restrict__ list, int tw0, int slabPlanes, int nch,
                   float2* __restrict__ grid) {
  const int t = list[blockIdx.x];
  const int tx = t % g.ntx, ty = (t / g.ntx) % g.nty, tw = t / (g.ntx * g.nty);
  const int xm = threadIdx.x % kTX, ym = threadIdx.x / kTX;
  for (int c = 0; c < nch; ++c)
#pragma unroll
    for (int pl = 0; pl < kTW; ++pl)
      grid[slab_index(g, nch, slabPlanes, c, (tw - tw0) * kTW + pl, ty * kTY + ym, tx * kTX + xm)] =
          make_float2(0.f, 0.f);
}

}  // namespace bippb200
