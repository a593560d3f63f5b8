// Pruned inverse 2-D FFT of the fine-grid planes, in place, as two passes of batched
// 1-D Stockham transforms (sm_100a).
//
// The w-sum reads, of every (channel, plane) array of ny x nx cells, only the Na x Nb
// outputs at the pixel lattice: pixel (a, b) takes the output at frequency
// ((a - Na/2) mod ny, (b - Nb/2) mod nx). (The reference's transform is neonufft's
// type-3 plan, src/gpu/nufft.hpp:198-210; this path's lattice form of it needs, per
// w-plane, only these cells.) Pass 1 transforms every row (along x, length nx) and keeps the Nb outputs the
// pixels read, written in place to the row's first Nb cells; pass 2 transforms those Nb
// columns (along y, length ny) and keeps Na outputs, written in place to the column's
// first Na cells. Cell (a, b) of the array then holds the 2-D inverse transform at pixel
// (a, b). A full 2-D transform reads and writes every cell in each of its passes; here a
// plane is read once, Nb/nx of it written, and only those columns read and (Na/ny of
// them) written again.
//
// A line (row or column) of n values is transformed by T threads of a CTA by the
// self-sorting Stockham algorithm: the stage of radix R that follows stages of total
// radix p takes, for butterfly b (0 <= b < n/R, k = b mod p), the inputs x[b + j n/R],
// multiplies input j by exp(2 pi i j k / (p R)), applies a length-R DFT and writes output
// j to y[(b - k) R + k + j p]; after the last stage the line is in natural order. The
// first stage reads its inputs straight from global memory and the last writes the kept
// outputs straight back; the stages between exchange through shared memory in place
// (every thread reads all of its inputs, the block synchronises, then every thread
// writes). Shared-memory slots are padded (the stride-R writes of a stage otherwise fall
// into a few banks; FftBlockPad). Butterfly additions are packed FP32x2. Sign convention: exp(+2 pi i jk/n), unnormalised, as
// an inverse cuFFT transform.
#pragma once

#include "common.cuh"

namespace bippb200 {

constexpr int kFftMaxStages = 4;
constexpr int kFftMaxValues = 16;   // complex values a thread holds in a stage

// One batched 1-D pass: the transform of length n, its stages and the launch shape.
struct FftLinePlan {
  int n;                         // transform length
  int nout;                      // outputs kept (the crop around frequency zero)
  int ns;                        // stages
  int radix[kFftMaxStages];      // radix of each stage
  int threads;                   // threads per line
  int lines;                     // lines per CTA
  int lineStride;                // shared-memory slots per line (padded)
};

// Which lines of a slab [channel][plane][y][x] a pass transforms.
struct FftLines {
  float2* data;
  long long nLines;              // channels x planes used x lines per plane
  int linesPerPlane;             // rows: ny; columns: Nb
  int planesUsed, slabPlanes;    // planes transformed / planes per channel in the slab
  long long planeStride;         // cells per plane
  long long lineStep;            // offset between consecutive lines (rows: nx; columns: 1)
  long long elemStep;            // offset between the values of a line (rows: 1; columns: nx)
};

__host__ __device__ __forceinline__ int fft_pad(int i) { return i + (i >> 4); }

// multiply by i
__device__ __forceinline__ float2 fft_mul_i(float2 z) { return mk(-z.y, z.x); }

// z exp(2 pi i m / 16) for m in [0, 16); m is a constant after unrolling
__device__ __forceinline__ float2 fft_rot16(float2 z, int m) {
  constexpr float c1 = 0.9238795325112867f, s1 = 0.3826834323650898f, h = 0.7071067811865476f;
  switch (m & 15) {
    case 0: return z;
    case 1: return mk(c1 * z.x - s1 * z.y, s1 * z.x + c1 * z.y);
    case 2: return mk(h * (z.x - z.y), h * (z.x + z.y));
    case 3: return mk(s1 * z.x - c1 * z.y, c1 * z.x + s1 * z.y);
    case 4: return mk(-z.y, z.x);
    case 5: return mk(-s1 * z.x - c1 * z.y, c1 * z.x - s1 * z.y);
    case 6: return mk(-h * (z.x + z.y), h * (z.x - z.y));
    case 7: return mk(-c1 * z.x - s1 * z.y, s1 * z.x - c1 * z.y);
    case 8: return mk(-z.x, -z.y);
    case 9: return mk(-c1 * z.x + s1 * z.y, -s1 * z.x - c1 * z.y);
    case 10: return mk(-h * (z.x - z.y), -h * (z.x + z.y));
    case 11: return mk(-s1 * z.x + c1 * z.y, -c1 * z.x - s1 * z.y);
    case 12: return mk(z.y, -z.x);
    case 13: return mk(s1 * z.x + c1 * z.y, -c1 * z.x + s1 * z.y);
    case 14: return mk(h * (z.x + z.y), h * (z.y - z.x));
    default: return mk(c1 * z.x + s1 * z.y, -s1 * z.x + c1 * z.y);
  }
}

// complex a + b and a - b as packed FP32x2 instructions (a - b = b (-1) + a, one rounding,
// the same value as two scalar subtractions)
__device__ __forceinline__ float2 fft_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 fft_sub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.f, -1.f), a); }

__device__ __forceinline__ void fft_dft2(float2& a, float2& b) {
  const float2 t = a;
  a = fft_add(t, b);
  b = fft_sub(t, b);
}

// X_k = sum_j x_j exp(2 pi i jk / 4)
__device__ __forceinline__ void fft_dft4(float2& x0, float2& x1, float2& x2, float2& x3) {
  const float2 a = fft_add(x0, x2), b = fft_sub(x0, x2), c = fft_add(x1, x3), t = fft_sub(x1, x3);
  x0 = fft_add(a, c);
  x2 = fft_sub(a, c);
  // b +- i t
  x1 = mk(b.x - t.y, b.y + t.x);
  x3 = mk(b.x + t.y, b.y - t.x);
}

// odd radix by the symmetric form: s_j = x_j + x_{R-j}, d_j = x_j - x_{R-j};
// X_k = x_0 + sum_j cos(2 pi jk/R) s_j + i sum_j sin(2 pi jk/R) d_j, X_{R-k} its mirror
template <int R>
__device__ __forceinline__ void fft_dft_odd(float2 (&x)[R], const float (&cs)[R], const float (&sn)[R]) {
  constexpr int H = (R - 1) / 2;
  float2 s[H + 1], d[H + 1];
  float2 x0 = x[0];
#pragma unroll
  for (int j = 1; j <= H; ++j) {
    s[j] = fft_add(x[j], x[R - j]);
    d[j] = fft_sub(x[j], x[R - j]);
    x0 = fft_add(x0, s[j]);
  }
#pragma unroll
  for (int k = 1; k <= H; ++k) {
    float2 A = x[0], B = mk(0.f, 0.f);
#pragma unroll
    for (int j = 1; j <= H; ++j) {
      const int m = (j * k) % R;
      A.x = fmaf(cs[m], s[j].x, A.x);
      A.y = fmaf(cs[m], s[j].y, A.y);
      B.x = fmaf(sn[m], d[j].x, B.x);
      B.y = fmaf(sn[m], d[j].y, B.y);
    }
    x[k] = mk(A.x - B.y, A.y + B.x);
    x[R - k] = mk(A.x + B.y, A.y - B.x);
  }
  x[0] = x0;
}

template <int R> __device__ __forceinline__ void fft_dft(float2 (&x)[R]) {
  if constexpr (R == 2) {
    fft_dft2(x[0], x[1]);
  } else if constexpr (R == 4) {
    fft_dft4(x[0], x[1], x[2], x[3]);
  } else if constexpr (R == 3) {
    const float cs[3] = {1.f, -0.5f, -0.5f};
    const float sn[3] = {0.f, 0.8660254037844387f, -0.8660254037844387f};
    fft_dft_odd<3>(x, cs, sn);
  } else if constexpr (R == 5) {
    const float cs[5] = {1.f, 0.30901699437494745f, -0.8090169943749473f, -0.8090169943749473f,
                         0.30901699437494745f};
    const float sn[5] = {0.f, 0.9510565162951535f, 0.5877852522924732f, -0.5877852522924732f,
                         -0.9510565162951535f};
    fft_dft_odd<5>(x, cs, sn);
  } else if constexpr (R == 7) {
    const float cs[7] = {1.f, 0.6234898018587336f, -0.22252093395631434f, -0.900968867902419f,
                         -0.900968867902419f, -0.22252093395631434f, 0.6234898018587336f};
    const float sn[7] = {0.f, 0.7818314824680298f, 0.9749279121818236f, 0.43388373911755823f,
                         -0.43388373911755823f, -0.9749279121818236f, -0.7818314824680298f};
    fft_dft_odd<7>(x, cs, sn);
  } else {
    // R = R1 R2 (8 = 2 x 4, 16 = 4 x 4): with n = R2 n1 + n2 and k = k1 + R1 k2,
    // X_k = sum_n2 exp(2 pi i n2 k2 / R2) exp(2 pi i n2 k1 / R) [DFT_R1 over n1 of x_{R2 n1 + n2}]_k1
    static_assert(R == 8 || R == 16, "radix");
    constexpr int R1 = R == 8 ? 2 : 4, R2 = 4;
    float2 Y[R2][R1];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
      float2 y[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) y[n1] = x[R2 * n1 + n2];
      if constexpr (R1 == 2) fft_dft2(y[0], y[1]);
      else fft_dft4(y[0], y[1], y[2], y[3]);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) Y[n2][k1] = fft_rot16(y[k1], (16 / R) * n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      float2 z0 = Y[0][k1], z1 = Y[1][k1], z2 = Y[2][k1], z3 = Y[3][k1];
      fft_dft4(z0, z1, z2, z3);
      x[k1] = z0;
      x[k1 + R1] = z1;
      x[k1 + 2 * R1] = z2;
      x[k1 + 3 * R1] = z3;
    }
  }
}

// Multiply input j (j = 1 .. R-1) of a butterfly by its twiddle w_j = exp(2 pi i j k / (P R))
// = tw[j m]: w_1 (and, for R >= 8, w_4) from the table, the others as products at most
// three deep (w_2 = w_1^2, w_3 = w_2 w_1, w_8 = w_4^2, w_12 = w_8 w_4, w_{4a+b} = w_{4a} w_b),
// so each carries a few roundings rather than the up to R - 1 of a power chain; applied as
// formed, so only w_1..w_3 and one w_{4a} are held.
template <int R>
__device__ __forceinline__ void fft_apply_twiddles(float2 (&v)[R], const float2* __restrict__ tw, int m) {
  const float2 w1 = __ldg(&tw[m]);
  v[1] = cmul(v[1], w1);
  if constexpr (R > 2) {
    const float2 w2 = cmul(w1, w1);
    v[2] = cmul(v[2], w2);
    if constexpr (R > 3) {
      const float2 w3 = cmul(w2, w1);
      v[3] = cmul(v[3], w3);
      if constexpr (R > 4) {
        float2 w4a = R >= 8 ? __ldg(&tw[4 * m]) : cmul(w2, w2);   // w_4, then w_8, w_12
        const float2 w4 = w4a;
#pragma unroll
        for (int a4 = 4; a4 < R; a4 += 4) {
          if (a4 > 4) w4a = a4 == 8 ? cmul(w4, w4) : cmul(w4a, w4);
          v[a4] = cmul(v[a4], w4a);
          if (a4 + 1 < R) v[a4 + 1] = cmul(v[a4 + 1], cmul(w4a, w1));
          if (a4 + 2 < R) v[a4 + 2] = cmul(v[a4 + 2], cmul(w4a, w2));
          if (a4 + 3 < R) v[a4 + 3] = cmul(v[a4 + 3], cmul(w4a, w3));
        }
      }
    }
  }
}

// Shared-memory slots of a line. The general layout pads one slot per 16 (fft_pad). Lines
// of N = 256 c (radices c, 16, 16, c odd) use a block layout instead: slot(i) = i + c
// floor(i / B), B = 16 c, under which every access of the three stages is a per-butterfly
// base plus a compile-time offset and stays free of bank conflicts: stage 1 writes
// c b + j -> c b + c floor(b / 16) + j; stages 2 and 3 read b + j B (b < B) -> b + j (B + c);
// stage 2 writes 16 c q + k + j c (q = floor(b / c), k = b mod c) -> (B + c) q + k + j c, and
// a half-warp's 16 consecutive b then fall in 16 distinct bank pairs.
template <int N, int... Rs> struct FftBlockPad {
  static constexpr int radix[sizeof...(Rs)] = {Rs...};
  static constexpr bool on = sizeof...(Rs) == 3 && radix[1] == 16 && radix[2] == 16 && (radix[0] & 1) == 1;
  static constexpr int c = radix[0], B = 16 * radix[0];
};

// One stage of radix R over the line of this thread's group (see the file comment); N the
// line length, P the product of the earlier radices, MODE 0 first, 1 middle, 2 last; ES the
// compile-time stride between a line's values in global memory (1 for rows; 0 takes the
// runtime es); offsets within one (channel, plane) array fit 32 bits; BP the block slot
// layout (FftBlockPad) when on, with its c.
template <int R, int MODE, int N, int P, int ES, bool BP, int BPC>
__device__ __forceinline__ void fft_stage(const FftLinePlan& pl, int t, bool active, float2* __restrict__ lp, int es,
                                          float2* __restrict__ sl, const float2* __restrict__ tw) {
  constexpr bool first = MODE == 0, last = MODE == 2;
  constexpr int MB = kFftMaxValues / R;   // butterflies per thread (the plan's thread count ensures enough)
  constexpr int Nr = N / R, twStep = N / (P * R);
  constexpr int BPB = 16 * BPC;           // block of the block layout
  const int T = pl.threads;
  const int st = ES > 0 ? ES : es;
  float2 v[MB][R];
#pragma unroll
  for (int q = 0; q < MB; ++q) {
    const int b = t + q * T;
    if (b < Nr) {
#pragma unroll
      for (int j = 0; j < R; ++j) {
        const int i = b + j * Nr;
        if constexpr (first) v[q][j] = active ? lp[i * st] : mk(0.f, 0.f);
        else if constexpr (BP) v[q][j] = sl[b + j * (BPB + BPC)];   // Nr == B in stages 2 and 3
        else v[q][j] = sl[fft_pad(i)];
      }
    }
  }
  // in place: every read of the line's buffer precedes every write (the last stage writes
  // global memory only, whose inputs the first stage read before its closing barrier)
  if constexpr (!first && !last) __syncthreads();
#pragma unroll
  for (int q = 0; q < MB; ++q) {
    const int b = t + q * T;
    if (b < Nr) {
      const int k = b % P;
      if constexpr (P > 1) fft_apply_twiddles<R>(v[q], tw, k * twStep);
      fft_dft<R>(v[q]);
      if constexpr (last) {
        // in the last stage b < P, so output j is frequency i = b + j P. Cell d of the nout
        // kept ones holds frequency (d - h) mod N, h = nout / 2: i < nout - h goes to cell
        // i + h, i >= N - h to cell i - (N - h), the others are not kept. The j ranges of
        // both are found once per butterfly
        const int h = pl.nout >> 1, lo = pl.nout - h, hi = N - h;
        const int j1 = lo > b ? (lo - b + P - 1) / P : 0;
        const int j2 = hi > b ? (hi - b + P - 1) / P : 0;
        const int offLo = (b + h) * st, offHi = (b - hi) * st;
#pragma unroll
        for (int j = 0; j < R; ++j) {
          if (active && j < j1) lp[offLo + j * P * st] = v[q][j];
          else if (active && j >= j2) lp[offHi + j * P * st] = v[q][j];
        }
      } else {
        const int o = (b - k) * R + k;
        int base = 0;
        if constexpr (BP && P == 1) base = BPC * b + BPC * (b >> 4);   // stage 1: c b + c floor(b / 16)
        else if constexpr (BP) base = (BPB + BPC) * (b / BPC) + k;      // stage 2: (B + c) q + k
#pragma unroll
        for (int j = 0; j < R; ++j) {
          if constexpr (BP) sl[base + j * P] = v[q][j];
          else sl[fft_pad(o + j * P)] = v[q][j];
        }
      }
    }
  }
  if constexpr (!last) __syncthreads();
}

template <int S, int N, int P, int ES, bool BP, int BPC, int R, int... Rest>
__device__ __forceinline__ void fft_stages(const FftLinePlan& pl, int t, bool active, float2* __restrict__ lp, int es,
                                           float2* __restrict__ sl, const float2* __restrict__ tw) {
  fft_stage<R, S == 0 ? 0 : (sizeof...(Rest) == 0 ? 2 : 1), N, P, ES, BP, BPC>(pl, t, active, lp, es, sl, tw);
  if constexpr (sizeof...(Rest) > 0)
    fft_stages<S + 1, N, P * R, ES, BP, BPC, Rest...>(pl, t, active, lp, es, sl, tw);
}

// The pass over lines of N = the product of the radices Rs (at least two stages).
// LINE_FAST: consecutive threads take consecutive lines (the column pass: a warp reads
// 32-byte row segments of 4 adjacent columns); otherwise consecutive threads take
// consecutive butterflies of one line (the row pass: contiguous row segments).
// tw[m] = exp(2 pi i m / N), m < N. Launch: lines x threads threads, lines x lineStride
// float2 of dynamic shared memory, ceil(nLines / lines) CTAs.
template <bool LINE_FAST, int... Rs>
__global__ void __launch_bounds__(512, 2) fft_lines_kernel(FftLinePlan pl, FftLines L, const float2* __restrict__ tw) {
  static_assert(sizeof...(Rs) >= 2, "two stages at least");
  constexpr int N = (Rs * ...);
  extern __shared__ float2 fft_smem[];
  const int T = pl.threads, G = pl.lines;
  const int tid = threadIdx.x;
  const int g = LINE_FAST ? tid % G : tid / T;
  const int t = LINE_FAST ? tid / G : tid % T;
  const long long line = (long long)blockIdx.x * G + g;
  const bool active = line < L.nLines;
  long long base = 0;
  if (active) {
    const long long o = line / L.linesPerPlane;
    const int li = (int)(line - o * L.linesPerPlane);
    const int c = (int)(o / L.planesUsed), pj = (int)(o - (long long)c * L.planesUsed);
    base = ((long long)c * L.slabPlanes + pj) * L.planeStride + (long long)li * L.lineStep;
  }
  // rows: unit stride (compile time); columns: the row length
  using BPad = FftBlockPad<N, Rs...>;
  fft_stages<0, N, 1, LINE_FAST ? 0 : 1, BPad::on, BPad::c, Rs...>(pl, t, active, L.data + base, (int)L.elemStep,
                                                                   fft_smem + (size_t)g * pl.lineStride, tw);
}

using FftLinesKernel = void (*)(FftLinePlan, FftLines, const float2*);

// Compiled radix sequences: the power of two 2^a (a = 4..9) as 4 x 4, 8 x 4, 16 x 4,
// 16 x 8, 16 x 16, 16 x 8 x 4, or one odd radix 3, 5 or 7 followed by 16, 8 x 4, 16 x 4,
// 16 x 8, 16 x 16, 16 x 8 x 4. Null when the sequence has no compiled kernel (the caller
// then transforms with cuFFT).
inline FftLinesKernel fft_lines_kernel_for(const int* radix, int ns, bool lineFast) {
  struct Entry {
    int r[4];
    FftLinesKernel rows, cols;
  };
#define B2_FFT_ENTRY(...) {{__VA_ARGS__}, fft_lines_kernel<false, __VA_ARGS__>, fft_lines_kernel<true, __VA_ARGS__>}
#define B2_FFT_ODD(f)                                                                                          \
  B2_FFT_ENTRY(f, 16), B2_FFT_ENTRY(f, 8, 4), B2_FFT_ENTRY(f, 16, 4), B2_FFT_ENTRY(f, 16, 8),                 \
      B2_FFT_ENTRY(f, 16, 16), B2_FFT_ENTRY(f, 16, 8, 4)
  static const Entry table[] = {B2_FFT_ENTRY(4, 4),  B2_FFT_ENTRY(8, 4),      B2_FFT_ENTRY(16, 4),
                                B2_FFT_ENTRY(16, 8), B2_FFT_ENTRY(16, 16),    B2_FFT_ENTRY(16, 8, 4),
                                B2_FFT_ODD(3),       B2_FFT_ODD(5),           B2_FFT_ODD(7)};
#undef B2_FFT_ODD
#undef B2_FFT_ENTRY
  for (const Entry& e : table) {
    int m = 0;
    while (m < 4 && e.r[m] != 0) ++m;
    bool same = m == ns;
    for (int s = 0; same && s < ns; ++s) same = e.r[s] == radix[s];
    if (same) return lineFast ? e.cols : e.rows;
  }
  return nullptr;
}

}  // namespace bippb200
