// Type-3 NUFFT kernels for image synthesis on a pixel lattice (sm_100a).
//
// Target sum (the reference's exact definition, src/host/kernels/nuft_sum.cpp:9-31 with
// alpha = 1 after the 2 pi/wl uvw scaling of src/nufft_synthesis.cpp:151-155):
//     I_l(p) += Re sum_k c_lk exp(i (u_k l_p + v_k m_p + w_k n_p))
// Pixels lie on a lattice l = l0 + a A_l + b B_l, m = m0 + a A_m + b B_m (a slow, b
// fast), so the (l, m) part is a periodic type-1 transform in the folded phases
// x_k = u B_l + v B_m, y_k = u A_l + v A_m, and n enters as a 1-D type-3 axis:
//   spread (ES kernel) onto a grid [level][w-plane][y][x] -> 2-D FFT per plane ->
//   per-pixel sum over w-planes with exp(i n~_p t_j) -> deconvolve, Re, accumulate.
// Points are bucket-sorted by tile so each CTA accumulates one output tile in shared
// memory and writes it once (no global atomics on the grid).
#pragma once

#include "common.cuh"

namespace bippb200 {

constexpr int kTX = 16, kTY = 8, kTW = 8;        // output tile (cells): 128 (x, y) cells x 8 w-planes
constexpr int kMaxW = 9;                          // max kernel width: a support crosses at most one tile edge (W - 1 <= kTY)
constexpr int kMaxChan = 12;                      // max channels (levels x correction terms)

struct NufftGeom {
  // lattice
  double l0, m0, Al, Bl, Am, Bm;   // pixel (a,b): l = l0 + a Al + b Bl, m = m0 + a Am + b Bm
  int Na, Nb;                       // lattice extents (a slow)
  double nc;                        // centre of n
  double wc;                        // centre of w
  // fine grid
  int nx, ny, nw;                   // grid sizes (nx, ny periodic; nw linear)
  int jc;                           // w-grid index of t = 0
  double hx, hy, hw;                // grid spacings (x,y in radians per cell; w in w-units)
  double ihx, ihy, ihw;             // their reciprocals (per-point coordinates multiply)
  int W;                            // kernel width (cells)
  float beta;                       // ES kernel shape
  int ntx, nty, ntw;                // tile counts
};

// Fine-grid slab layout: cell (channel c, plane, y, x) of a slab of slabPlanes w-planes at
// ((c slabPlanes + plane) ny + y) nx + x, i.e. [channel][plane][y][x]: every (channel,
// plane) is one contiguous ny x nx array, transformed in place by the pruned two-pass FFT
// (fft_kernels.cuh: rows, then the kept columns), or by one batched 2-D cuFFT plan for
// grid sizes without a compiled pruned plan. (A [y][channel][plane][x] layout that let
// the pass along x skip the rows no pixel reads made cuFFT's strided pass along y three
// times slower than the whole 2-D transform.)
__host__ __device__ __forceinline__ long long slab_index(const NufftGeom& g, int nch, int slabPlanes, int c, int plane,
                                                       int y, int x) {
  (void)nch;
  return (((long long)c * slabPlanes + plane) * g.ny + y) * g.nx + x;
}

// ES kernel exp(beta (sqrt(1 - z^2) - 1)), |z| < 1
__device__ __forceinline__ float es_kernel(float z, float beta) {
  const float t = fmaf(-z, z, 1.0f);
  // the hardware square root (PTX sqrt.approx, relative error ~2^-23): the kernel values
  // enter 3xTF32 products (~2^-21) and a kernel that approximates the ideal one to eps
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(fmaxf(t, 0.0f)));
  return t > 0.0f ? __expf(beta * (r - 1.0f)) : 0.0f;
}

__device__ __forceinline__ double wrap_pi(double x) {
  // to [-pi, pi)
  const double twopi = 6.283185307179586476925286766559;
  const double inv_twopi = 0.15915494309189533576888376337251;
  return x - twopi * floor(x * inv_twopi + 0.5);
}

// grid coordinates of one point: first support cell and offset (gx - ix0) in FP32
struct PtCoord {
  int ix0, iy0, iw0;
  float dx, dy, dw;
};

// not inlined: the count and scatter passes must compute bit-identical keys
static __device__ __noinline__ PtCoord point_coord(const NufftGeom& g, double u, double v, double w) {
  const double x = u * g.Bl + v * g.Bm;
  const double y = u * g.Al + v * g.Am;
  const double gx = wrap_pi(x) * g.ihx;
  const double gy = wrap_pi(y) * g.ihy;
  const double gw = (w - g.wc) * g.ihw + g.jc;
  const double half = 0.5 * g.W;
  PtCoord c;
  c.ix0 = (int)ceil(gx - half);
  c.iy0 = (int)ceil(gy - half);
  c.iw0 = (int)ceil(gw - half);
  c.dx = (float)(gx - c.ix0);
  c.dy = (float)(gy - c.iy0);
  c.dw = (float)(gw - c.iw0);
  c.iw0 = min(max(c.iw0, 0), g.nw - g.W);
  return c;
}

// phase of a point at the lattice origin, reduced to [-pi, pi) in FP64
__device__ __forceinline__ double point_phase(const NufftGeom& g, double u, double v, double w) {
  const double x = u * g.Bl + v * g.Bm;
  const double y = u * g.Al + v * g.Am;
  // exp(i (u l0 + v m0 + x Nb/2 + y Na/2 + w nc)): the Nb/2, Na/2 shifts centre the modes
  double ph = u * g.l0 + v * g.m0 + w * g.nc;
  ph = wrap_pi(ph) + wrap_pi(x * (double)(g.Nb / 2)) + wrap_pi(y * (double)(g.Na / 2));
  return wrap_pi(ph);
}

static __device__ __noinline__ int tile_key(const NufftGeom& g, const PtCoord& c) {
  int ix = c.ix0 % g.nx; if (ix < 0) ix += g.nx;
  int iy = c.iy0 % g.ny; if (iy < 0) iy += g.ny;
  const int tx = ix / kTX, ty = iy / kTY, tw = c.iw0 / kTW;
  // crossing bits: support [i0, i0+W-1] crosses into the next tile
  const int bx = ((ix % kTX) + g.W - 1) >= kTX;
  const int by = ((iy % kTY) + g.W - 1) >= kTY;
  const int bw = ((c.iw0 % kTW) + g.W - 1) >= kTW;
  const int tile = (tw * g.nty + ty) * g.ntx + tx;
  return tile * 8 + (bx | (by << 1) | (bw << 2));
}

// sorted point record
struct __align__(16) PtRec {
  int ix0, iy0, iw0;
  float dx, dy, dw;
  int pad0, pad1;
};

// ---------------------------------------------------------------------------------------
// point sources: either pipeline form (antenna coordinates + VV lower triangle) or
// collect/get form (per-baseline float uvw + values)
// ---------------------------------------------------------------------------------------
struct PipelinePoints {
  // step s of the batch, pair (r >= s') of kept antennas
  int nSteps;
  const int* nred;            // [steps]
  const int* idx;             // [steps][Nmax]
  const double* antUVW;       // [steps][nAnt][3] antenna UVW coordinates (m)
  const double* uvwScale;     // [steps] 2 pi / wl
  const long long* pairOffset;// [steps+1] prefix of n(n+1)/2
  int Nmax, nAnt;
  const float2* vv;           // [steps][levels][Nmax*Nmax] lower triangle, column-major
  long long vvStepStride, vvLevelStride;
  int levels;
  int stepBase;               // first step of this chunk within the batch (for pairOffset)
};

struct BaselinePoints {
  long long n;                // number of points
  const float* uvw;           // [3][ld] float, in metres (scaled by uvwScale)
  long long lduvw;
  double uvwScale;            // 2 pi / wl (or 1)
  const float2* values;       // [channels][ldv]
  long long ldv;
  int levels;
};

static __device__ __noinline__ void pair_from_linear(long long t, int n, int& r, int& s) {
  // t enumerates the lower triangle column by column: column s holds rows s..n-1
  // offset(s) = s n - s (s - 1) / 2
  double nn = (double)n + 0.5;
  int sc = (int)floor(nn - sqrt(nn * nn - 2.0 * (double)t));
  if (sc < 0) sc = 0;
  if (sc > n - 1) sc = n - 1;
  long long off = (long long)sc * n - (long long)sc * (sc - 1) / 2;
  while (off > t) { --sc; off = (long long)sc * n - (long long)sc * (sc - 1) / 2; }
  while (true) {
    long long nxt = (long long)(sc + 1) * n - (long long)(sc + 1) * sc / 2;
    if (sc + 1 < n && nxt <= t) { ++sc; off = nxt; } else break;
  }
  s = sc;
  r = sc + (int)(t - off);
}

// pass 1: keys of pipeline points -> counts
static __global__ void __launch_bounds__(256, 8) pipeline_count_kernel(NufftGeom g, PipelinePoints P, long long total, int* __restrict__ counts,
                                      const long long* __restrict__ chunkPairOffset) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    // locate step by binary search in chunkPairOffset[0..nSteps]
    int lo = 0, hi = P.nSteps;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (chunkPairOffset[mid] <= t) lo = mid; else hi = mid;
    }
    const int st = lo;
    const int n = P.nred[st];
    int r, s;
    pair_from_linear(t - chunkPairOffset[st], n, r, s);
    if (r == s) continue;  // zero baseline: added analytically (Re of the trace of VV)
    const int ar = P.idx[(long long)st * P.Nmax + r], as = P.idx[(long long)st * P.Nmax + s];
    const double* U = P.antUVW + (long long)st * P.nAnt * 3;
    const double sc = P.uvwScale[st];
    double u = (U[ar * 3 + 0] - U[as * 3 + 0]) * sc;
    double v = (U[ar * 3 + 1] - U[as * 3 + 1]) * sc;
    double w = (U[ar * 3 + 2] - U[as * 3 + 2]) * sc;
    // only the real part of the image is kept, and a point and its mirror (-u, -v, -w,
    // conjugate value) have the same real part: every point is taken with w >= 0, so the
    // w-grid spans [0, max w] instead of [-max w, max w]
    const bool flip = w < 0.0;
    if (flip) { u = -u; v = -v; w = -w; }
    const PtCoord c = point_coord(g, u, v, w);
    atomicAdd(counts + tile_key(g, c), 1);
  }
}

// pass 2: scatter records + values (channel-major: vals[ch][sortedIndex])
static __global__ void pipeline_scatter_kernel(NufftGeom g, PipelinePoints P, long long total, int* __restrict__ cursor,
                                        const long long* __restrict__ chunkPairOffset, PtRec* __restrict__ rec,
                                        float2* __restrict__ vals, long long valStride, int sincos64, int nchAll) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = P.nSteps;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (chunkPairOffset[mid] <= t) lo = mid; else hi = mid;
    }
    const int st = lo;
    const int n = P.nred[st];
    int r, s;
    pair_from_linear(t - chunkPairOffset[st], n, r, s);
    if (r == s) continue;  // zero baseline: added analytically (Re of the trace of VV)
    const int ar = P.idx[(long long)st * P.Nmax + r], as = P.idx[(long long)st * P.Nmax + s];
    const double* U = P.antUVW + (long long)st * P.nAnt * 3;
    const double sc = P.uvwScale[st];
    double u = (U[ar * 3 + 0] - U[as * 3 + 0]) * sc;
    double v = (U[ar * 3 + 1] - U[as * 3 + 1]) * sc;
    double w = (U[ar * 3 + 2] - U[as * 3 + 2]) * sc;
    // only the real part of the image is kept, and a point and its mirror (-u, -v, -w,
    // conjugate value) have the same real part: every point is taken with w >= 0, so the
    // w-grid spans [0, max w] instead of [-max w, max w]
    const bool flip = w < 0.0;
    if (flip) { u = -u; v = -v; w = -w; }
    const PtCoord c = point_coord(g, u, v, w);
    const int key = tile_key(g, c);
    const int pos = atomicAdd(cursor + key, 1);
    if (pos < 0 || pos >= valStride) continue;  // keys of both passes agree; never taken
    PtRec pr;
    pr.ix0 = c.ix0; pr.iy0 = c.iy0; pr.iw0 = c.iw0;
    pr.dx = c.dx; pr.dy = c.dy; pr.dw = c.dw;
    pr.pad0 = 0; pr.pad1 = 0;
    rec[pos] = pr;
    const double ph = point_phase(g, u, v, w);
    float sn, cs;
    if (sincos64) { double s64, c64; sincos(ph, &s64, &c64); sn = (float)s64; cs = (float)c64; }
    else sincosf((float)ph, &sn, &cs);
    const float wgt = (r == s) ? 1.0f : 2.0f;   // lower triangle stands for (r,s) and (s,r)
    const float2* vvb = P.vv + (long long)st * P.vvStepStride + r + (long long)s * P.Nmax;
    for (int l = 0; l < P.levels; ++l) {
      float2 a = vvb[(long long)l * P.vvLevelStride];
      if (flip) a.y = -a.y;
      vals[(long long)pos * nchAll + l] = make_float2(wgt * (a.x * cs - a.y * sn), wgt * (a.x * sn + a.y * cs));
    }
  }
}

// zeroAcc[l] += sum_steps sum_r Re VV_l[r, r] (the r == s points skipped by the scatter)
static __global__ void vv_trace_kernel(int nSteps, int levels, const int* __restrict__ nred, const float2* __restrict__ vv,
                                       long long vvStepStride, long long vvLevelStride, int Nmax,
                                       double* __restrict__ zeroAcc) {
  __shared__ double red[32];
  const int b = blockIdx.x / levels, l = blockIdx.x % levels;
  if (b >= nSteps) return;
  const int n = nred[b];
  const float2* m = vv + (long long)b * vvStepStride + (long long)l * vvLevelStride;
  double acc = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) acc += (double)m[r + (long long)r * Nmax].x;
  acc = block_sum(acc, red);
  if (threadIdx.x == 0) atomicAdd(zeroAcc + l, acc);
}

// collect/get form: per-baseline uvw (float, metres) and values; optional first-order
// lattice-residual channels (values * u/su, values * v/sv)
static __global__ void baseline_count_kernel(NufftGeom g, BaselinePoints P, int* __restrict__ counts) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < P.n; t += (long long)gridDim.x * blockDim.x) {
    double u = (double)P.uvw[t] * P.uvwScale;
    double v = (double)P.uvw[t + P.lduvw] * P.uvwScale;
    double w = (double)P.uvw[t + 2 * P.lduvw] * P.uvwScale;
    if (u == 0.0 && v == 0.0 && w == 0.0) continue;  // zero baseline: added analytically
    if (w < 0.0) { u = -u; v = -v; w = -w; }         // folded to w >= 0 (real image)
    atomicAdd(counts + tile_key(g, point_coord(g, u, v, w)), 1);
  }
}

static __global__ void baseline_scatter_kernel(NufftGeom g, BaselinePoints P, int* __restrict__ cursor,
                                        PtRec* __restrict__ rec, float2* __restrict__ vals, long long valStride,
                                        int sincos64, int corrTerms, double su, double sv,
                                        double* __restrict__ zeroAcc, int nchAll) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < P.n; t += (long long)gridDim.x * blockDim.x) {
    double u = (double)P.uvw[t] * P.uvwScale;
    double v = (double)P.uvw[t + P.lduvw] * P.uvwScale;
    double w = (double)P.uvw[t + 2 * P.lduvw] * P.uvwScale;
    if (u == 0.0 && v == 0.0 && w == 0.0) {
      // exp(i 0) = 1 at every pixel: Re(value) adds to the whole image
      for (int l = 0; l < P.levels; ++l) atomicAdd(zeroAcc + l, (double)P.values[(long long)l * P.ldv + t].x);
      continue;
    }
    // the image is the real part: the mirror (-u, -v, -w, conjugate value) contributes the
    // same, so every point is taken with w >= 0 (the first-order channels follow, since
    // Re(i d u q) is unchanged under u -> -u, q -> conj q)
    const bool flip = w < 0.0;
    if (flip) { u = -u; v = -v; w = -w; }
    const PtCoord c = point_coord(g, u, v, w);
    const int pos = atomicAdd(cursor + tile_key(g, c), 1);
    if (pos < 0 || pos >= valStride) continue;  // keys of both passes agree; never taken
    PtRec pr;
    pr.ix0 = c.ix0; pr.iy0 = c.iy0; pr.iw0 = c.iw0;
    pr.dx = c.dx; pr.dy = c.dy; pr.dw = c.dw;
    pr.pad0 = 0; pr.pad1 = 0;
    rec[pos] = pr;
    const double ph = point_phase(g, u, v, w);
    float sn, cs;
    if (sincos64) { double s64, c64; sincos(ph, &s64, &c64); sn = (float)s64; cs = (float)c64; }
    else sincosf((float)ph, &sn, &cs);
    for (int l = 0; l < P.levels; ++l) {
      float2 a = P.values[(long long)l * P.ldv + t];
      if (flip) a.y = -a.y;
      const float2 q = make_float2(a.x * cs - a.y * sn, a.x * sn + a.y * cs);
      vals[(long long)pos * nchAll + l] = q;
      if (corrTerms) {
        const float fu = (float)(u / su), fv = (float)(v / sv);
        vals[(long long)pos * nchAll + P.levels + l] = make_float2(q.x * fu, q.y * fu);
        vals[(long long)pos * nchAll + 2 * P.levels + l] = make_float2(q.x * fv, q.y * fv);
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// exclusive scan (3 phases) of int counts -> int offsets
// ---------------------------------------------------------------------------------------
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;   // per thread

static __global__ void scan_partial_kernel(const int* __restrict__ in, int* __restrict__ out, long long n,
                                    int* __restrict__ blockSums) {
  __shared__ int warpSums[32];
  const long long base = (long long)blockIdx.x * kScanThreads * kScanItems;
  int vals[kScanItems];
  int tsum = 0;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const long long idx = base + (long long)threadIdx.x * kScanItems + i;
    vals[i] = (idx < n) ? in[idx] : 0;
    tsum += vals[i];
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int incl = tsum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  if (lane == 31) warpSums[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int ws = warpSums[lane];
    int wi = ws;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, wi, o);
      if (lane >= o) wi += t;
    }
    warpSums[lane] = wi - ws;
    if (lane == 31) blockSums[blockIdx.x] = wi;
  }
  __syncthreads();
  int run = warpSums[wid] + incl - tsum;
#pragma unroll
  for (int i = 0; i < kScanItems; ++i) {
    const long long idx = base + (long long)threadIdx.x * kScanItems + i;
    if (idx < n) out[idx] = run;
    run += vals[i];
  }
}

static __global__ void scan_blocksums_kernel(int* __restrict__ blockSums, int nBlocks, int* __restrict__ total) {
  // single block, sequential chunks
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nBlocks; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = (i < nBlocks) ? blockSums[i] : 0;
    // block inclusive scan
    __shared__ int tmp[1024];
    tmp[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < blockDim.x; o <<= 1) {
      const int t = (threadIdx.x >= o) ? tmp[threadIdx.x - o] : 0;
      __syncthreads();
      tmp[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nBlocks) blockSums[i] = carry + tmp[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += tmp[threadIdx.x];
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

static __global__ void scan_add_kernel(int* __restrict__ out, long long n, const int* __restrict__ blockSums,
                                int* __restrict__ out2) {
  const long long base = (long long)blockIdx.x * kScanThreads * kScanItems;
  const int add = blockSums[blockIdx.x];
  for (int i = threadIdx.x; i < kScanThreads * kScanItems; i += blockDim.x) {
    const long long idx = base + i;
    if (idx < n) {
      const int v = out[idx] + add;
      out[idx] = v;
      if (out2) out2[idx] = v;
    }
  }
}

// ---------------------------------------------------------------------------------------
// spreading: one CTA per work item (an output tile of the current w-slab, or one part of
// a heavily loaded tile); one warp per point, lanes over the W^3 support cells, shared-
// memory accumulation with a bank swizzle, one write of the tile (global atomics only for
// tiles split into several parts).
// ---------------------------------------------------------------------------------------
constexpr int kSpreadThreads = 256;
constexpr int kTileCells = kTX * kTY * kTW;

static_assert(kMaxW - 1 <= kTX && kMaxW - 1 <= kTY && kMaxW - 1 <= kTW, "tile smaller than a kernel support");

struct SpreadItem {
  int tile;    // tile index (tw * nty + ty) * ntx + tx
  int part;    // part index
  int nparts;  // number of parts of this tile
  int load;    // points of the tile (all parts)
};

// The 27 (source tile, crossing bits) key ranges whose points reach tile (tx, ty, tw).
struct TileRanges {
  int beg[27], end[27];
  int n;
};

__device__ __forceinline__ void tile_ranges(const NufftGeom& g, const int* __restrict__ offsets, int tx, int ty, int tw,
                                            TileRanges& R) {
  R.n = 0;
  for (int d = 0; d < 8; ++d) {
    const int dx = d & 1, dy = (d >> 1) & 1, dw = (d >> 2) & 1;
    const int stw = tw - dw;
    if (stw < 0) continue;
    const int stx = (tx - dx + g.ntx) % g.ntx;
    const int sty = (ty - dy + g.nty) % g.nty;
    const int stile = (stw * g.nty + sty) * g.ntx + stx;
    for (int bits = 0; bits < 8; ++bits) {
      if ((bits & d) != d) continue;
      const int key = stile * 8 + bits;
      R.beg[R.n] = offsets[key];
      R.end[R.n] = offsets[key + 1];
      ++R.n;
    }
  }
}

static __global__ void tile_load_kernel(NufftGeom g, const int* __restrict__ offsets, int* __restrict__ load) {
  const int ntiles = g.ntx * g.nty * g.ntw;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int tx = t % g.ntx, ty = (t / g.ntx) % g.nty, tw = t / (g.ntx * g.nty);
    TileRanges R;
    tile_ranges(g, offsets, tx, ty, tw, R);
    int s = 0;
    for (int i = 0; i < R.n; ++i) s += R.end[i] - R.beg[i];
    load[t] = s;
  }
}

// spreading parts of each tile (ceil(load / cap), 0 when empty) and whether the tile has
// to be cleared before spreading (empty, or spread in several parts that accumulate)
static __global__ void tile_parts_kernel(int ntiles, const int* __restrict__ load, int cap, int* __restrict__ parts,
                                         int* __restrict__ clearFlag, int* __restrict__ splitTiles) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int np = (load[t] + cap - 1) / cap;
    parts[t] = np;
    clearFlag[t] = (np != 1) ? 1 : 0;
    if (np > 1) atomicAdd(splitTiles, 1);
  }
}

// sort keys of the spreading work items for the load-ordered schedule: slab index in the
// high bits (items of a slab stay one contiguous range), then the item's points in
// descending order (heaviest first)
static __global__ void item_key_kernel(int nItems, const SpreadItem* __restrict__ items, int tilesPerSlab,
                                       unsigned* __restrict__ keys) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nItems; i += gridDim.x * blockDim.x) {
    const SpreadItem it = items[i];
    const long long lo = (long long)it.load * it.part / it.nparts, hi = (long long)it.load * (it.part + 1) / it.nparts;
    const long long pts = hi - lo;
    const unsigned n = (unsigned)(pts < 0xFFFFF ? pts : 0xFFFFF);
    keys[i] = ((unsigned)(it.tile / tilesPerSlab) << 20) | (0xFFFFFu - n);
  }
}

// tiles to clear, compacted in tile order (offsets from an exclusive scan of the flags)
static __global__ void clear_list_kernel(int ntiles, const int* __restrict__ clearFlag, const int* __restrict__ off,
                                         int* __restrict__ list) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x)
    if (clearFlag[t]) list[off[t]] = t;
}

// work items of every tile at its exclusive-scan offset
static __global__ void item_fill_kernel(int ntiles, const int* __restrict__ load, const int* __restrict__ parts,
                                        const int* __restrict__ itemOff, SpreadItem* __restrict__ items) {
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < ntiles; t += gridDim.x * blockDim.x) {
    const int np = parts[t];
    for (int q = 0; q < np; ++q) items[itemOff[t] + q] = SpreadItem{t, q, np, load[t]};
  }
}

// swizzled cell index inside the tile: x is rotated by W * (y / 2) so that the W x W
// footprint of a point covers distinct banks
__device__ __forceinline__ int tile_cell(int x, int y, int w, int W) {
  return (w * kTY + y) * kTX + ((x + W * (y >> 1)) & (kTX - 1));
}

template <int CH, int W>
__global__ void __launch_bounds__(kSpreadThreads)
spread_warp_kernel(NufftGeom g, const int* __restrict__ offsets, const PtRec* __restrict__ rec,
                   const float2* __restrict__ vals, long long valStride, int nch, const SpreadItem* __restrict__ items,
                   int tw0, int slabPlanes, float2* __restrict__ grid) {
  extern __shared__ float sacc[];   // [nch][2][kTileCells]  (re, im planes)
  __shared__ int rBeg[27], rPre[28];
  const SpreadItem it = items[blockIdx.x];
  const int tx = it.tile % g.ntx, ty = (it.tile / g.ntx) % g.nty, tw = it.tile / (g.ntx * g.nty);
  const int twl = tw - tw0;
  for (int i = threadIdx.x; i < nch * 2 * kTileCells; i += blockDim.x) sacc[i] = 0.f;
  if (threadIdx.x == 0) {
    TileRanges R;
    tile_ranges(g, offsets, tx, ty, tw, R);
    int pre = 0;
    for (int i = 0; i < R.n; ++i) {
      rBeg[i] = R.beg[i];
      rPre[i] = pre;
      pre += R.end[i] - R.beg[i];
    }
    for (int i = R.n; i < 28; ++i) rPre[i] = pre;
  }
  __syncthreads();
  const int x0 = tx * kTX, y0 = ty * kTY, w0 = tw * kTW;
  constexpr int W3 = W * W * W;
  constexpr int nIter = (W3 + 31) / 32;
  const float invHalf = 2.0f / (float)W;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  // lane-constant support offsets (x, y, w) of the cells this lane covers, packed 8 bits each
  unsigned cellOff[nIter];
#pragma unroll
  for (int i = 0; i < nIter; ++i) {
    const int c = i * 32 + lane;
    const int x = c % W, y = (c / W) % W, w = c / (W * W);
    cellOff[i] = (c < W3) ? (unsigned)(x | (y << 8) | (w << 16)) : 0xffffffffu;
  }
  // this part's window of the concatenated ranges, dealt to the warps round robin
  const int lo = (int)((long long)it.load * it.part / it.nparts);
  const int hi = (int)((long long)it.load * (it.part + 1) / it.nparts);
  int ri = 0;
  for (int q = lo + warp; q < hi; q += nwarp) {
    while (q >= rPre[ri + 1]) ++ri;
    const int p = rBeg[ri] + (q - rPre[ri]);
    const PtRec pr = rec[p];
    int lx = pr.ix0 - x0;
    lx = ((lx % g.nx) + g.nx) % g.nx;
    if (lx > g.nx / 2) lx -= g.nx;
    int ly = pr.iy0 - y0;
    ly = ((ly % g.ny) + g.ny) % g.ny;
    if (ly > g.ny / 2) ly -= g.ny;
    const int lw = pr.iw0 - w0;
    float kx = 0.f, ky = 0.f, kw = 0.f;
    if (lane < W) {
      kx = es_kernel(((float)lane - pr.dx) * invHalf, g.beta);
      ky = es_kernel(((float)lane - pr.dy) * invHalf, g.beta);
      kw = es_kernel(((float)lane - pr.dw) * invHalf, g.beta);
    }
    float2 v[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) v[c] = (c < nch) ? vals[(long long)p * nch + c] : make_float2(0.f, 0.f);
#pragma unroll
    for (int i = 0; i < nIter; ++i) {
      const unsigned o = cellOff[i];
      const int x = o & 0xff, y = (o >> 8) & 0xff, w = (o >> 16) & 0xff;
      const float wx = __shfl_sync(0xffffffffu, kx, x & 31);
      const float wy = __shfl_sync(0xffffffffu, ky, y & 31);
      const float ww = __shfl_sync(0xffffffffu, kw, w & 31);
      const int cx = lx + x, cy = ly + y, cw = lw + w;
      if (o != 0xffffffffu && (unsigned)cx < (unsigned)kTX && (unsigned)cy < (unsigned)kTY &&
          (unsigned)cw < (unsigned)kTW) {
        const float k = wx * wy * ww;
        const int cell = tile_cell(cx, cy, cw, W);
#pragma unroll
        for (int ch = 0; ch < CH; ++ch) {
          if (ch < nch) {
            atomicAdd(&sacc[(ch * 2) * kTileCells + cell], k * v[ch].x);
            atomicAdd(&sacc[(ch * 2 + 1) * kTileCells + cell], k * v[ch].y);
          }
        }
      }
    }
  }
  __syncthreads();
  // write the tile into the slab layout (slab_index), plane relative to the slab start
  for (int i = threadIdx.x; i < nch * kTileCells; i += blockDim.x) {
    const int c = i / kTileCells, rem = i % kTileCells;
    const int lw = rem / (kTX * kTY), ly = (rem / kTX) % kTY, lx = rem % kTX;
    const int cell = tile_cell(lx, ly, lw, W);
    const float2 val = make_float2(sacc[(c * 2) * kTileCells + cell], sacc[(c * 2 + 1) * kTileCells + cell]);
    const long long off = slab_index(g, nch, slabPlanes, c, twl * kTW + lw, y0 + ly, x0 + lx);
    if (it.nparts == 1) {
      grid[off] = val;
    } else if (val.x != 0.f || val.y != 0.f) {
      atomicAdd(&grid[off].x, val.x);
      atomicAdd(&grid[off].y, val.y);
    }
  }
}

// ---------------------------------------------------------------------------------------
// w-sum: acc[ch][p] += sum_{planes j of slab} F[ch][j][a'][b'] exp(i n~_p t_j)
// ---------------------------------------------------------------------------------------
// CH: channels held in registers (4, or kMaxChan for more); with 4 channels the planes are
// read 4 at a time (their 16 loads issued together), with more one at a time (registers),
// while the FP64 phase recurrence runs in order
template <int CH, int kWsumUnroll = (CH <= 4 ? 4 : 1)>
static __global__ void __launch_bounds__(256) wsum_kernel(NufftGeom g, const float2* __restrict__ F, int nch,
                                                           int slabPlanes, int jFirst, int planesUsed,
                                                           const double* __restrict__ nTilde /*[P]*/,
                                                           float2* __restrict__ acc, long long accStride,
                                                           int pruned) {
  const long long P = (long long)g.Na * g.Nb;
  const long long planeStride = (long long)g.ny * g.nx;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(p / g.Nb), b = (int)(p % g.Nb);
    // pixel (a, b) reads frequency ((a - Na/2) mod ny, (b - Nb/2) mod nx): that cell of a
    // full transform, or cell (a, b) of the pruned one (fft_kernels.cuh)
    int ap = a, bp = b;
    if (!pruned) {
      ap = a - g.Na / 2; if (ap < 0) ap += g.ny;
      bp = b - g.Nb / 2; if (bp < 0) bp += g.nx;
    }
    const double nt = nTilde[p];
    // exp(i nt t_j), t_j = (j - jc) hw; recurrence in FP64
    double s0, c0, sd, cd;
    sincos(nt * (double)(jFirst - g.jc) * g.hw, &s0, &c0);
    sincos(nt * g.hw, &sd, &cd);
    double er = c0, ei = s0;
    float2 sum[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) sum[c] = make_float2(0.f, 0.f);
    const float2* Fp = F + slab_index(g, nch, slabPlanes, 0, 0, ap, bp);   // channel 0, plane 0
    for (int j0 = 0; j0 < planesUsed; j0 += kWsumUnroll) {
      float2 f[kWsumUnroll][CH];
#pragma unroll
      for (int u = 0; u < kWsumUnroll; ++u)
#pragma unroll
        for (int c = 0; c < CH; ++c)
          f[u][c] = (c < nch && j0 + u < planesUsed)
                        ? Fp[((long long)c * slabPlanes + (j0 + u)) * planeStride]
                        : make_float2(0.f, 0.f);
#pragma unroll
      for (int u = 0; u < kWsumUnroll; ++u) {
        const float fr = (float)er, fi = (float)ei;
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          sum[c].x += f[u][c].x * fr - f[u][c].y * fi;
          sum[c].y += f[u][c].x * fi + f[u][c].y * fr;
        }
        const double nr = er * cd - ei * sd;
        ei = er * sd + ei * cd;
        er = nr;
      }
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      if (c < nch) {
        float2 o = acc[(long long)c * accStride + p];
        o.x += sum[c].x;
        o.y += sum[c].y;
        acc[(long long)c * accStride + p] = o;
      }
    }
  }
}

// image_l[p] += Re(decon_p exp(i wc n~_p) (acc_l + i dl_p su acc_u + i dm_p sv acc_v)); the
// two extra channel groups carry the first-order lattice-residual terms when enabled.
static __global__ void finalize_kernel(long long P, int levels, const float2* __restrict__ acc, long long accStride,
                                const double* __restrict__ decon, const double* __restrict__ nTilde, double wc,
                                int corrTerms, const double* __restrict__ dl, const double* __restrict__ dm, double su,
                                double sv, float* __restrict__ image, long long ldImage,
                                const double* __restrict__ zeroAcc) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    double sn, cs;
    sincos(wc * nTilde[p], &sn, &cs);
    const double dc = decon[p];
    const double cfx = dc * cs, cfy = dc * sn;
    for (int l = 0; l < levels; ++l) {
      double2 a = to_d(acc[(long long)l * accStride + p]);
      if (corrTerms) {
        const double2 au = to_d(acc[(long long)(levels + l) * accStride + p]);
        const double2 av = to_d(acc[(long long)(2 * levels + l) * accStride + p]);
        const double tu = dl[p] * su, tv = dm[p] * sv;
        a.x -= tu * au.y + tv * av.y;
        a.y += tu * au.x + tv * av.x;
      }
      image[(long long)l * ldImage + p] += (float)(cfx * a.x - cfy * a.y + zeroAcc[l]);
    }
  }
}

// per-pixel deconvolution factor hx hy hw / (psi_x(b') psi_y(a') psi_w(n~)) with
// psi(xi) = (W h / 2) int_{-1}^{1} es(z) cos(xi W h z / 2) dz (Gauss-Legendre)
static __global__ void decon_kernel(NufftGeom g, const double* __restrict__ nTilde, const double* __restrict__ qz,
                             const double* __restrict__ qw, int nq, double* __restrict__ decon) {
  const long long P = (long long)g.Na * g.Nb;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < P; p += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(p / g.Nb), b = (int)(p % g.Nb);
    const double bp = (double)(b - g.Nb / 2), ap = (double)(a - g.Na / 2);
    const double nt = nTilde[p];
    const double hxh = 0.5 * g.W * g.hx, hyh = 0.5 * g.W * g.hy, hwh = 0.5 * g.W * g.hw;
    double fx = 0, fy = 0, fw = 0;
    for (int q = 0; q < nq; ++q) {
      const double z = qz[q];
      const double t = 1.0 - z * z;
      const double k = t > 0 ? exp((double)g.beta * (sqrt(t) - 1.0)) * qw[q] : 0.0;
      fx += k * cos(bp * hxh * z);
      fy += k * cos(ap * hyh * z);
      fw += k * cos(nt * hwh * z);
    }
    fx *= hxh; fy *= hyh; fw *= hwh;
    decon[p] = g.hx * g.hy * g.hw / (fx * fy * fw);
  }
}

// ---------------------------------------------------------------------------------------
// direct sum out_l[p] += Re sum_k in_lk exp(i alpha (x_p u_k + y_p v_k + z_p w_k))
// FP64 phase argument reduced to [-pi, pi) before the sine/cosine.
// ---------------------------------------------------------------------------------------
constexpr int kDirectThreads = 256;
constexpr int kDirectChunk = 256;

template <typename TC, typename C, typename TO, int CH>
__global__ void __launch_bounds__(kDirectThreads)
direct_sum_kernel(double alpha, long long nIn, const C* __restrict__ input, long long ldIn,
                  const TC* __restrict__ u, const TC* __restrict__ v, const TC* __restrict__ w, long long nOut,
                  const TC* __restrict__ x, const TC* __restrict__ y, const TC* __restrict__ z, TO* __restrict__ out,
                  long long ldOut, int nch, int fp64Trig) {
  __shared__ double su[kDirectChunk], sv[kDirectChunk], sw[kDirectChunk];
  __shared__ C sval[CH][kDirectChunk];
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const bool active = p < nOut;
  const double xp = active ? (double)x[p] * alpha : 0.0;
  const double yp = active ? (double)y[p] * alpha : 0.0;
  const double zp = active ? (double)z[p] * alpha : 0.0;
  double acc[CH];
#pragma unroll
  for (int c = 0; c < CH; ++c) acc[c] = 0.0;
  const double twopi = 6.283185307179586476925286766559;
  const double inv2pi = 1.0 / twopi;
  // blockIdx.y takes one slice of the inputs (whole chunks); slices add their partial
  // sums atomically when the inputs are split
  const long long per = ((nIn + gridDim.y - 1) / gridDim.y + kDirectChunk - 1) / kDirectChunk * kDirectChunk;
  const long long kBegin = (long long)blockIdx.y * per;
  const long long kEnd = (kBegin + per < nIn) ? kBegin + per : nIn;
  for (long long k0 = kBegin; k0 < kEnd; k0 += kDirectChunk) {
    const int nk = (kEnd - k0 < (long long)kDirectChunk) ? (int)(kEnd - k0) : kDirectChunk;
    __syncthreads();
    for (int i = threadIdx.x; i < nk; i += blockDim.x) {
      su[i] = (double)u[k0 + i];
      sv[i] = (double)v[k0 + i];
      sw[i] = (double)w[k0 + i];
#pragma unroll
      for (int c = 0; c < CH; ++c)
        if (c < nch) sval[c][i] = input[(long long)c * ldIn + k0 + i];
    }
    __syncthreads();
    if (active) {
      for (int i = 0; i < nk; ++i) {
        double ph = fma(xp, su[i], fma(yp, sv[i], zp * sw[i]));
        ph = fma(-twopi, rint(ph * inv2pi), ph);
        double s, cs;
        if (fp64Trig) {
          sincos(ph, &s, &cs);
        } else {
          float sf, cf;
          __sincosf((float)ph, &sf, &cf);
          s = sf;
          cs = cf;
        }
#pragma unroll
        for (int c = 0; c < CH; ++c) {
          if (c < nch) {
            const C a = sval[c][i];
            acc[c] = fma((double)a.x, cs, fma(-(double)a.y, s, acc[c]));
          }
        }
      }
    }
  }
  if (active) {
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      if (c < nch) {
        if (gridDim.y > 1)
          atomicAdd(&out[(long long)c * ldOut + p], (TO)acc[c]);
        else
          out[(long long)c * ldOut + p] += (TO)acc[c];
      }
    }
  }
}

// Grid of direct_sum_kernel: one thread per output; when the outputs fill fewer than
// ctasPerSm CTAs per SM, the inputs are split over blockIdx.y (slices of at least 4096
// inputs) so that few pixels over many baselines still fill the GPU.
inline dim3 direct_sum_grid(long long nOut, long long nIn, int smCount, int ctasPerSm) {
  const long long bx = (nOut + kDirectThreads - 1) / kDirectThreads;
  const long long target = (long long)ctasPerSm * (smCount > 0 ? smCount : 148);
  long long by = 1;
  if (bx < target) {
    by = (target + bx - 1) / bx;
    const long long maxSlices = nIn / 4096 > 1 ? nIn / 4096 : 1;
    by = by < maxSlices ? by : maxSlices;
    by = by < 65535 ? by : 65535;
  }
  return dim3((unsigned)bx, (unsigned)by, 1);
}

// scale[c] = the largest |Re| or |Im| of channel c over the sorted points (vals[p nch + c],
// p < *total), as FP32 bits (non-negative floats order as unsigned integers); scale[] is
// zeroed before the launch
static __global__ void value_scale_kernel(const int* __restrict__ total, const float2* __restrict__ vals, int nch,
                                          unsigned* __restrict__ scale) {
  __shared__ unsigned smax[kMaxChan];
  if (threadIdx.x < kMaxChan) smax[threadIdx.x] = 0u;
  __syncthreads();
  const long long n = *total;
  float m[kMaxChan];
#pragma unroll
  for (int c = 0; c < kMaxChan; ++c) m[c] = 0.f;
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
#pragma unroll
    for (int c = 0; c < kMaxChan; ++c) {
      if (c < nch) {
        const float2 v = vals[p * nch + c];
        m[c] = fmaxf(m[c], fmaxf(fabsf(v.x), fabsf(v.y)));
      }
    }
  }
#pragma unroll
  for (int c = 0; c < kMaxChan; ++c)
    if (c < nch) atomicMax(&smax[c], __float_as_uint(m[c]));
  __syncthreads();
  if (threadIdx.x < nch) atomicMax(scale + threadIdx.x, smax[threadIdx.x]);
}

}  // namespace bippb200
