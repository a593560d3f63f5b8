// Batched generalized Hermitian eigensolver kernels (sm_100a).
//
// Pipeline per matrix b of a batch (sizes vary per matrix after flagging):
//   prep_kernel        flag non-zero rows/cols of S, compact S -> A (working precision),
//                      Gram G_ij = sinc(2|p_i-p_j|/wl) -> G (FP64)       [src/eigensolver.cpp:148-207,
//                                                                          src/host/gram_matrix.cpp:23-56]
//   cholesky_kernel    G = L L^H in FP64                                   [LAPACK potrf inside ?hegv]
//   trinv_kernel       Linv = L^-1 in FP64, rounded to working precision
//   gemm_kernel        C = Linv S Linv^H (two triangular products)         [hegst]
//   hetrd_kernel       C = Q T Q^H, T real tridiagonal (Householder)        [hetrd]
//   tridiag_kernel     eigenpairs of T in FP64: bisection + twisted factorisation
//   backtransform      Y = Q Z                                              [unmtr]
//   gemm_kernel        X = Linv^H Y                                         [trsm back-transform]
// One CTA owns one matrix in the sequential stages; matrices live in HBM with
// leading dimension Nmax (the batch's padded size).
#pragma once

#include "common.cuh"

namespace bippb200 {

constexpr int kPrepThreads = 512;

// ------------------------------------------------------------------------------------
// prep: flagging, compaction, Gram
// ------------------------------------------------------------------------------------
// mode 0: eigh_gram flag test |s|^2 > eps (src/eigensolver.cpp:150-158)
// mode 1: eigh flag test |Re| >= eps || |Im| >= eps (src/eigensolver.cpp:59-68)
template <typename T>
__global__ void __launch_bounds__(kPrepThreads)
prep_kernel(int nBeam, const typename Cplx<T>::type* __restrict__ S, long long sStride, int lds,
            const double* __restrict__ xyz, long long xyzStride, int ldxyz,
            const double* __restrict__ wl, int mode, T eps, int withGram, int Nmax,
            int* __restrict__ idxOut, int* __restrict__ nredOut, long long* __restrict__ nvisOut,
            typename Cplx<T>::type* __restrict__ A, double2* __restrict__ G, int* __restrict__ status,
            int doFlag, int doCompact, int batchOffset) {
  using C = typename Cplx<T>::type;
  extern __shared__ int smem_i[];
  int* flags = smem_i;                 // [Nmax]
  int* idx = smem_i + Nmax;            // [Nmax]
  __shared__ long long red_ll[32];
  __shared__ int s_nred;
  const int b = blockIdx.x;                 // matrix within this launch
  const int bg = b + batchOffset;           // matrix within the flag/index arrays
  const C* Sb = S + b * sStride;
  int* idxB = idxOut + (long long)bg * Nmax;
  if (doFlag) {
    for (int i = threadIdx.x; i < nBeam; i += blockDim.x) flags[i] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    long long cnt = 0;
    int bad = 0;
    for (int col = warp; col < nBeam; col += nwarp) {
      for (int row = col + lane; row < nBeam; row += 32) {
        C v = Sb[row + (long long)col * lds];
        if (!isfinite(v.x) || !isfinite(v.y)) bad = 1;
        bool nz = (mode == 0) ? (flag_norm(v) > eps) : (fabs(v.x) >= eps || fabs(v.y) >= eps);
        if (nz) {
          flags[row] = 1;
          flags[col] = 1;
          cnt += (row == col) ? 1 : 2;
        }
      }
    }
    long long nvis = block_sum(cnt, red_ll);
    // a non-finite entry fails the flag test; it is an error only where its row and
    // column are both kept, i.e. where it enters the reduced matrix (the reference's
    // LAPACK call then returns info != 0)
    if (__syncthreads_or(bad)) {
      int kept = 0;
      for (int col = warp; col < nBeam; col += nwarp) {
        if (!flags[col]) continue;
        for (int row = col + lane; row < nBeam; row += 32) {
          const C v = Sb[row + (long long)col * lds];
          if ((!isfinite(v.x) || !isfinite(v.y)) && flags[row]) kept = 1;
        }
      }
      if (kept) atomicOr(status + bg, (int)kStatusNonFinite);
    }
    __syncthreads();
    // compaction scan (warp 0)
    if (warp == 0) {
      const int per = (nBeam + 31) / 32;
      const int beg = lane * per, end = min(nBeam, beg + per);
      int c = 0;
      for (int i = beg; i < end; ++i) c += flags[i];
      int incl = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int t = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += t;
      }
      int pos = incl - c;
      for (int i = beg; i < end; ++i)
        if (flags[i]) idx[pos++] = i;
      if (lane == 31) s_nred = incl;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      nredOut[bg] = s_nred;
      nvisOut[bg] = nvis;
    }
    for (int i = threadIdx.x; i < s_nred; i += blockDim.x) idxB[i] = idx[i];
  } else {
    if (threadIdx.x == 0) s_nred = nredOut[bg];
    __syncthreads();
    for (int i = threadIdx.x; i < s_nred; i += blockDim.x) idx[i] = idxB[i];
    __syncthreads();
  }
  if (!doCompact) return;
  const int nr = s_nred;

  // compacted full Hermitian matrix from the lower triangle of S
  C* Ab = A + (long long)b * Nmax * Nmax;
  for (long long e = threadIdx.x; e < (long long)nr * nr; e += blockDim.x) {
    const int r = (int)(e % nr), c = (int)(e / nr);
    const int ir = idx[r], ic = idx[c];
    C v;
    if (r >= c) {
      v = Sb[ir + (long long)ic * lds];
    } else {
      v = cconj(Sb[ic + (long long)ir * lds]);
    }
    if (r == c) v.y = 0;
    Ab[r + (long long)c * Nmax] = v;
  }
  if (withGram) {
    const double* xb = xyz + bg * xyzStride;
    const double w = wl[bg];
    double2* Gb = G + (long long)b * Nmax * Nmax;
    for (long long e = threadIdx.x; e < (long long)nr * nr; e += blockDim.x) {
      const int r = (int)(e % nr), c = (int)(e / nr);
      if (r < c) continue;
      double g = 1.0;
      if (r != c) {
        const int ir = idx[r], ic = idx[c];
        const double dx = xb[ir] - xb[ic];
        const double dy = xb[ir + ldxyz] - xb[ic + ldxyz];
        const double dz = xb[ir + 2 * ldxyz] - xb[ic + 2 * ldxyz];
        const double x = 2.0 * sqrt(dx * dx + dy * dy + dz * dz) / w;
        g = (x != 0.0) ? sinpi(x) / (3.14159265358979323846 * x) : 1.0;
      }
      if (withGram == 2)
        reinterpret_cast<double*>(G)[(long long)b * Nmax * Nmax + r + (long long)c * Nmax] = g;
      else
        Gb[r + (long long)c * Nmax] = make_double2(g, 0.0);
    }
  }
}

// ------------------------------------------------------------------------------------
// Cholesky (FP64 complex, lower, in place), blocked right-looking, NB = 32
// ------------------------------------------------------------------------------------
constexpr int kCholNB = 32;
constexpr int kCholThreads = 256;
// shared memory: diagonal block D, its inverse Dinv, and two 64-row panel tiles
template <typename E>
constexpr size_t chol_smem() { return (size_t)(2 * kCholNB + 128) * (kCholNB + 1) * sizeof(E); }
constexpr size_t kCholSmem = chol_smem<double2>();

// FP64 element helpers: E = double2 (complex Hermitian G) or double (real symmetric G,
// identity beamforming)
template <typename E> __device__ __forceinline__ E e_zero();
template <> __device__ __forceinline__ double2 e_zero<double2>() { return make_double2(0.0, 0.0); }
template <> __device__ __forceinline__ double e_zero<double>() { return 0.0; }
__device__ __forceinline__ double e_re(double2 a) { return a.x; }
__device__ __forceinline__ double e_re(double a) { return a; }
__device__ __forceinline__ double2 e_real(double2, double v) { return make_double2(v, 0.0); }
__device__ __forceinline__ double e_real(double, double v) { return v; }
__device__ __forceinline__ double2 e_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double e_scale(double a, double s) { return a * s; }
__device__ __forceinline__ double2 e_neg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double e_neg(double a) { return -a; }
// acc -= a conj(b)
__device__ __forceinline__ void e_sub_mulc(double2& acc, double2 a, double2 b) {
  acc.x -= a.x * b.x + a.y * b.y;
  acc.y -= a.y * b.x - a.x * b.y;
}
__device__ __forceinline__ void e_sub_mulc(double& acc, double a, double b) { acc -= a * b; }
// acc -= a b
__device__ __forceinline__ void e_sub_mul(double2& acc, double2 a, double2 b) {
  acc.x -= a.x * b.x - a.y * b.y;
  acc.y -= a.x * b.y + a.y * b.x;
}
__device__ __forceinline__ void e_sub_mul(double& acc, double a, double b) { acc -= a * b; }
// acc += a conj(b)
__device__ __forceinline__ void e_add_mulc(double2& acc, double2 a, double2 b) {
  acc.x += a.x * b.x + a.y * b.y;
  acc.y += a.y * b.x - a.x * b.y;
}
__device__ __forceinline__ void e_add_mulc(double& acc, double a, double b) { acc += a * b; }
// acc += a b
__device__ __forceinline__ void e_add_mul(double2& acc, double2 a, double2 b) { cfma(acc, a, b); }
__device__ __forceinline__ void e_add_mul(double& acc, double a, double b) { acc += a * b; }
// a / d
__device__ __forceinline__ double2 e_div(double2 a, double2 d) {
  const double den = d.x * d.x + d.y * d.y;
  return make_double2((a.x * d.x + a.y * d.y) / den, (a.y * d.x - a.x * d.y) / den);
}
__device__ __forceinline__ double e_div(double a, double d) { return a / d; }

// Panel rows below the diagonal block are X = A L_kk^-H with L_kk^-1 formed in shared
// memory (as the triangular inverse does per block), a register-tiled product that keeps
// the kernel at three CTAs per SM in the real case.
template <typename E>
__global__ void __launch_bounds__(kCholThreads, sizeof(E) == 8 ? 4 : 1)
cholesky_kernel(E* __restrict__ G, const int* __restrict__ nred, int Nmax, int* __restrict__ status,
                const int* __restrict__ order = nullptr) {
  const int b = order ? order[blockIdx.x] : blockIdx.x;
  const int n = nred[b];
  E* Gb = G + (long long)b * Nmax * Nmax;
  extern __shared__ __align__(16) unsigned char chol_raw[];
  E* chol_smem = reinterpret_cast<E*>(chol_raw);
  E (*D)[kCholNB + 1] = reinterpret_cast<E (*)[kCholNB + 1]>(chol_smem);
  E (*Dinv)[kCholNB + 1] = reinterpret_cast<E (*)[kCholNB + 1]>(chol_smem + kCholNB * (kCholNB + 1));
  E (*Pi)[kCholNB + 1] = reinterpret_cast<E (*)[kCholNB + 1]>(chol_smem + 2 * kCholNB * (kCholNB + 1));
  E (*Pj)[kCholNB + 1] = reinterpret_cast<E (*)[kCholNB + 1]>(chol_smem + (2 * kCholNB + 64) * (kCholNB + 1));
  __shared__ int s_bad;
  if (threadIdx.x == 0) s_bad = 0;
  const int tid = threadIdx.x;
  const E zero = e_zero<E>();
  for (int k0 = 0; k0 < n; k0 += kCholNB) {
    const int kb = min(kCholNB, n - k0);
    // 1. load diagonal block (lower)
    __syncthreads();
    for (int e = tid; e < kCholNB * kCholNB; e += blockDim.x) {
      const int r = e % kCholNB, c = e / kCholNB;
      D[r][c] = (r < kb && c < kb && r >= c) ? Gb[(k0 + r) + (long long)(k0 + c) * Nmax] : zero;
    }
    __syncthreads();
    // 2. unblocked factorisation in smem
    for (int j = 0; j < kb; ++j) {
      if (tid == 0) {
        double djj = e_re(D[j][j]);
        if (!(djj > 0.0)) {
          s_bad = 1;
          djj = 1e-300;
        }
        D[j][j] = e_real(zero, sqrt(djj));
      }
      __syncthreads();
      const double inv = 1.0 / e_re(D[j][j]);
      for (int r = j + 1 + tid; r < kb; r += blockDim.x) D[r][j] = e_scale(D[r][j], inv);
      __syncthreads();
      // trailing update inside the block: D[r][c] -= D[r][j] conj(D[c][j]), j < c <= r
      for (int e = tid; e < kb * kb; e += blockDim.x) {
        const int r = e % kb, c = e / kb;
        if (c > j && r >= c) {
          E t = D[r][c];
          e_sub_mulc(t, D[r][j], D[c][j]);
          D[r][c] = t;
        }
      }
      __syncthreads();
    }
    // 3. write back diagonal block
    for (int e = tid; e < kb * kb; e += blockDim.x) {
      const int r = e % kb, c = e / kb;
      if (r >= c) Gb[(k0 + r) + (long long)(k0 + c) * Nmax] = D[r][c];
    }
    // 4. Dinv = L_kk^-1 (lower; zero above the diagonal and outside kb): thread c forms
    // column c by forward substitution
    if (tid < kCholNB) {
      const int c = tid;
      for (int r = 0; r < kCholNB; ++r) {
        E acc = e_real(zero, r == c ? 1.0 : 0.0);
        if (r < kb && c < kb && r >= c) {
          for (int m = c; m < r; ++m) e_sub_mul(acc, D[r][m], Dinv[m][c]);
          Dinv[r][c] = e_div(acc, D[r][r]);
        } else {
          Dinv[r][c] = zero;
        }
      }
    }
    // 5. panel rows i >= k0+kb, 64 at a time: X = A L_kk^-H, X[i][c] = sum_m A[i][m] conj(Dinv[c][m])
    for (int p0 = k0 + kb; p0 < n; p0 += 64) {
      __syncthreads();
      for (int e = tid; e < 64 * kCholNB; e += blockDim.x) {
        const int r = e % 64, c = e / 64;
        Pi[r][c] = (p0 + r < n && c < kb) ? Gb[(p0 + r) + (long long)(k0 + c) * Nmax] : zero;
      }
      __syncthreads();
      const int tr = tid % 16, tc = tid / 16;  // rows tr + 16 a, columns tc + 16 c
      E acc[4][2];
#pragma unroll
      for (int a = 0; a < 4; ++a) acc[a][0] = acc[a][1] = zero;
      for (int m = 0; m < kb; ++m) {
        E pa[4], pb[2];
#pragma unroll
        for (int a = 0; a < 4; ++a) pa[a] = Pi[tr + 16 * a][m];
#pragma unroll
        for (int c = 0; c < 2; ++c) pb[c] = Dinv[tc + 16 * c][m];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 2; ++c) e_add_mulc(acc[a][c], pa[a], pb[c]);
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int i = p0 + tr + 16 * a, col = tc + 16 * c;
          if (i < n && col < kb) Gb[i + (long long)(k0 + col) * Nmax] = acc[a][c];
        }
    }
    __syncthreads();
    // 5. trailing update A[i,j] -= sum_m P[i,m] conj(P[j,m]) for j <= i, tiles 64x64
    const int t0 = k0 + kb;
    const int nt = n - t0;
    if (nt <= 0) continue;
    const int ntile = (nt + 63) / 64;
    for (int ti = 0; ti < ntile; ++ti) {
      for (int tj = 0; tj <= ti; ++tj) {
        const int i0 = t0 + ti * 64, j0 = t0 + tj * 64;
        __syncthreads();
        // the row panel of tile row ti is loaded once, the column panel per tile
        for (int e = tid; e < 64 * kCholNB; e += blockDim.x) {
          const int r = e % 64, c = e / 64;
          if (tj == 0) Pi[r][c] = (i0 + r < n && c < kb) ? Gb[(i0 + r) + (long long)(k0 + c) * Nmax] : zero;
          Pj[r][c] = (j0 + r < n && c < kb) ? Gb[(j0 + r) + (long long)(k0 + c) * Nmax] : zero;
        }
        __syncthreads();
        // each thread: 4x4 outputs; thread (tr, tc) in 16x16 grid
        const int tr = tid % 16, tc = tid / 16;
        E acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 4; ++c) acc[a][c] = zero;
        for (int m = 0; m < kb; ++m) {
          E pa[4], pb[4];
#pragma unroll
          for (int a = 0; a < 4; ++a) pa[a] = Pi[tr + 16 * a][m];
#pragma unroll
          for (int c = 0; c < 4; ++c) pb[c] = Pj[tc + 16 * c][m];
#pragma unroll
          for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int c = 0; c < 4; ++c) e_add_mulc(acc[a][c], pa[a], pb[c]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            const int i = i0 + tr + 16 * a, j = j0 + tc + 16 * c;
            if (i < n && j < n && j <= i) {
              E* p = Gb + i + (long long)j * Nmax;
              E v = *p;
              e_sub_mul(v, acc[a][c], e_real(zero, 1.0));
              *p = v;
            }
          }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0 && s_bad) atomicOr(status + b, (int)kStatusCholeskyNotPD);
}

// ------------------------------------------------------------------------------------
// triangular inverse of the lower Cholesky factor (FP64), output in working precision
// ------------------------------------------------------------------------------------
// FP64 value -> output element of Linv (complex or real, working precision)
__device__ __forceinline__ void store_conv(float2* p, double2 v) { *p = to_f(v); }
__device__ __forceinline__ void store_conv(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void store_conv(float* p, double v) { *p = (float)v; }
__device__ __forceinline__ void store_conv(double* p, double v) { *p = v; }

// Linv is computed block row by block row: Linv[I,I] = inv(L[I,I]);
// Linv[I,J] = -Linv[I,I] sum_{K=J}^{I-1} L[I,K] Linv[K,J]. The FP64 inverse goes to W64
// (read back for the later block rows) and, rounded, to LinvOut. E = double2 (complex)
// or double (real symmetric G); O = the matching working-precision output element.
template <typename E>
constexpr size_t trinv_smem() { return 3 * 32 * 33 * sizeof(E); }
constexpr size_t kTrinvSmem = trinv_smem<double2>();

template <typename E, typename O>
__global__ void __launch_bounds__(256, sizeof(E) == 8 ? 8 : 1)
trinv_kernel(const E* __restrict__ L, E* __restrict__ W64, O* __restrict__ LinvOut, const int* __restrict__ nred,
             int Nmax, const int* __restrict__ order = nullptr) {
  constexpr int NB = 32;
  const int b = order ? order[blockIdx.x] : blockIdx.x;
  const int n = nred[b];
  const E* Lb = L + (long long)b * Nmax * Nmax;
  E* Wb = W64 + (long long)b * Nmax * Nmax;
  O* Ob = LinvOut + (long long)b * Nmax * Nmax;
  extern __shared__ __align__(16) unsigned char trinv_raw[];
  E* trinv_smem_p = reinterpret_cast<E*>(trinv_raw);
  E (*Dinv)[NB + 1] = reinterpret_cast<E (*)[NB + 1]>(trinv_smem_p);
  E (*Ta)[NB + 1] = reinterpret_cast<E (*)[NB + 1]>(trinv_smem_p + NB * (NB + 1));
  E (*Tb)[NB + 1] = reinterpret_cast<E (*)[NB + 1]>(trinv_smem_p + 2 * NB * (NB + 1));
  const int tid = threadIdx.x;
  const E zero = e_zero<E>();
  const int nblk = (n + NB - 1) / NB;
  for (int I = 0; I < nblk; ++I) {
    const int i0 = I * NB, ib = min(NB, n - i0);
    __syncthreads();
    // load L_II into Ta (lower) and invert into Dinv by column forward substitution
    for (int e = tid; e < NB * NB; e += blockDim.x) {
      const int r = e % NB, c = e / NB;
      Ta[r][c] = (r < ib && c < ib && r >= c) ? Lb[(i0 + r) + (long long)(i0 + c) * Nmax] : zero;
    }
    __syncthreads();
    if (tid < NB) {
      const int c = tid;  // column c of the inverse
      for (int r = 0; r < NB; ++r) {
        E acc = e_real(zero, r == c ? 1.0 : 0.0);
        if (r < ib && c < ib && r >= c) {
          for (int m = c; m < r; ++m) e_sub_mul(acc, Ta[r][m], Dinv[m][c]);
          Dinv[r][c] = e_div(acc, Ta[r][r]);
        } else {
          Dinv[r][c] = zero;
        }
      }
    }
    __syncthreads();
    for (int e = tid; e < NB * NB; e += blockDim.x) {
      const int r = e % NB, c = e / NB;
      if (r < ib && c < ib) {
        const E v = (r >= c) ? Dinv[r][c] : zero;
        Wb[(i0 + r) + (long long)(i0 + c) * Nmax] = v;
        store_conv(Ob + (i0 + r) + (long long)(i0 + c) * Nmax, v);
      }
    }
    // strictly upper blocks J > I are zero (the GEMMs read whole tiles of Linv)
    for (long long e = tid; e < (long long)ib * (n - i0 - ib); e += blockDim.x) {
      const int r = (int)(e % ib), c = i0 + ib + (int)(e / ib);
      Wb[(i0 + r) + (long long)c * Nmax] = zero;
      store_conv(Ob + (i0 + r) + (long long)c * Nmax, zero);
    }
    // off-diagonal blocks J < I
    for (int J = 0; J < I; ++J) {
      const int j0 = J * NB;
      const int tr = tid % 16, tc = tid / 16;  // 16x16 threads, 2x2 outputs each
      E acc[2][2] = {{zero, zero}, {zero, zero}};
      for (int K = J; K < I; ++K) {
        const int k0 = K * NB;
        __syncthreads();
        for (int e = tid; e < NB * NB; e += blockDim.x) {
          const int r = e % NB, c = e / NB;
          Ta[r][c] = (r < ib) ? Lb[(i0 + r) + (long long)(k0 + c) * Nmax] : zero;
          Tb[r][c] = Wb[(k0 + r) + (long long)(j0 + c) * Nmax];
        }
        __syncthreads();
#pragma unroll 4
        for (int m = 0; m < NB; ++m) {
#pragma unroll
          for (int a = 0; a < 2; ++a)
#pragma unroll
            for (int c = 0; c < 2; ++c) e_add_mul(acc[a][c], Ta[tr + 16 * a][m], Tb[m][tc + 16 * c]);
        }
      }
      __syncthreads();
      // Tb <- acc
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < 2; ++c) Tb[tr + 16 * a][tc + 16 * c] = acc[a][c];
      __syncthreads();
      // out = -Dinv * Tb
      E o[2][2] = {{zero, zero}, {zero, zero}};
      for (int m = 0; m < NB; ++m) {
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int c = 0; c < 2; ++c) e_add_mul(o[a][c], Dinv[tr + 16 * a][m], Tb[m][tc + 16 * c]);
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const int r = tr + 16 * a, cc = tc + 16 * c;
          if (r < ib && j0 + cc < n) {
            const E v = e_neg(o[a][c]);
            Wb[(i0 + r) + (long long)(j0 + cc) * Nmax] = v;
            store_conv(Ob + (i0 + r) + (long long)(j0 + cc) * Nmax, v);
          }
        }
    }
  }
}

// ------------------------------------------------------------------------------------
// batched complex GEMM with triangular skipping, per-matrix sizes and k-ranges
// ------------------------------------------------------------------------------------
template <typename C>
struct GemmArgs {
  // A and B are complex C or, for the real-operand instantiations, real R (element strides)
  const void* A; long long strideA; int lda; int opA;   // opA 0: A[i,k]; 1: conj(A[k,i])
  const void* B; long long strideB; int ldb; int opB;   // opB 0: B[k,j]; 1: conj(B[j,k])
  C* Cm; long long strideC; int ldc;
  const int* n;           // per-matrix size
  int triA;               // 0 none; 1 opA(i,k)=0 for k>i; 2 opA(i,k)=0 for k<i
  int triB;               // 0 none; 1 opB(k,j)=0 for k>j; 2 opB(k,j)=0 for k<j
  int outMode;            // 0 full; 1 lower tiles + conj mirror; 2 lower tiles only (i>=j)
  const void* kscale; long long strideK;   // optional real per-k scale on opA columns
  const int* kbeg; const int* kend;        // optional per-(matrix,level) k range
  int levels;             // grid.z = batch * levels (levels >= 1)
  const int* colRange;    // optional [2 per matrix]: only output columns [lo, hi) are needed
  long long strideCLevel; // output stride per level
};

constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 8, kGemmThreads = 256;

// operand helpers: conj of a real value is itself; the product of a complex accumulator
// with real / complex operands
__device__ __forceinline__ float opconj(float a) { return a; }
__device__ __forceinline__ double opconj(double a) { return a; }
__device__ __forceinline__ float2 opconj(float2 a) { return cconj(a); }
__device__ __forceinline__ double2 opconj(double2 a) { return cconj(a); }
__device__ __forceinline__ float opscale(float a, float s) { return a * s; }
__device__ __forceinline__ double opscale(double a, double s) { return a * s; }
__device__ __forceinline__ float2 opscale(float2 a, float s) { return cscale(a, s); }
__device__ __forceinline__ double2 opscale(double2 a, double s) { return cscale(a, s); }
template <typename E> __device__ __forceinline__ E opzero();
template <> __device__ __forceinline__ float opzero<float>() { return 0.f; }
template <> __device__ __forceinline__ double opzero<double>() { return 0.0; }
template <> __device__ __forceinline__ float2 opzero<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 opzero<double2>() { return make_double2(0.0, 0.0); }
template <typename C> __device__ __forceinline__ void opfma(C& acc, C a, C b) { cfma(acc, a, b); }
__device__ __forceinline__ void opfma(float2& acc, float a, float2 b) { acc.x = fmaf(a, b.x, acc.x); acc.y = fmaf(a, b.y, acc.y); }
__device__ __forceinline__ void opfma(float2& acc, float2 a, float b) { acc.x = fmaf(a.x, b, acc.x); acc.y = fmaf(a.y, b, acc.y); }
__device__ __forceinline__ void opfma(double2& acc, double a, double2 b) { acc.x = fma(a, b.x, acc.x); acc.y = fma(a, b.y, acc.y); }
__device__ __forceinline__ void opfma(double2& acc, double2 a, double b) { acc.x = fma(a.x, b, acc.x); acc.y = fma(a.y, b, acc.y); }

// EA / EB: element types of A / B (C complex, or R real: Linv of a real Gram matrix)
template <typename C, typename R, typename EA = C, typename EB = C>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(GemmArgs<C> g) {
  const int z = blockIdx.z;
  const int b = z / g.levels, lvl = z % g.levels;
  const int n = g.n[b];
  const int i0 = blockIdx.y * kGemmBM, j0 = blockIdx.x * kGemmBN;
  if (i0 >= n || j0 >= n) return;
  if (g.outMode != 0 && j0 > i0 + kGemmBM - 1) return;
  if (g.colRange && (j0 + kGemmBN <= g.colRange[2 * b] || j0 >= g.colRange[2 * b + 1])) return;
  int kb = 0, ke = n;
  if (g.kbeg) {
    kb = g.kbeg[z];
    ke = g.kend[z];
  }
  // triangular limits
  if (g.triA == 1) ke = min(ke, i0 + kGemmBM);
  if (g.triA == 2) kb = max(kb, i0);
  if (g.triB == 1) ke = min(ke, j0 + kGemmBN);
  if (g.triB == 2) kb = max(kb, j0);
  const EA* A = static_cast<const EA*>(g.A) + b * g.strideA;
  const EB* B = static_cast<const EB*>(g.B) + b * g.strideB;
  C* Cm = g.Cm + b * g.strideC + lvl * g.strideCLevel;
  const R* ks = g.kscale ? reinterpret_cast<const R*>(g.kscale) + b * g.strideK : nullptr;

  // k-tiles of BK, double-buffered in shared memory; the next tile's global loads are
  // issued before the current tile is multiplied
  constexpr int BK = sizeof(C) == 8 ? 2 * kGemmBK : kGemmBK;
  constexpr int LPT = kGemmBM * BK / kGemmThreads;   // elements of A (and of B) per thread
  __shared__ EA As[2][BK][kGemmBM + 1];
  __shared__ EB Bs[2][BK][kGemmBN + 1];
  const int tid = threadIdx.x;
  const int tr = tid % 16, tc = tid / 16;
  C acc[4][4];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[a][c] = mk(R(0), R(0));
  EA ra[LPT];
  EB rb[LPT];
  auto load = [&](int k0) {
#pragma unroll
    for (int t = 0; t < LPT; ++t) {
      const int e = tid + t * kGemmThreads;
      int r, kk;
      if (g.opA == 0) { r = e % kGemmBM; kk = e / kGemmBM; } else { kk = e % BK; r = e / BK; }
      const int i = i0 + r, k = k0 + kk;
      EA v = opzero<EA>();
      if (i < n && k < ke) {
        v = (g.opA == 0) ? A[i + (long long)k * g.lda] : opconj(A[k + (long long)i * g.lda]);
        if (ks) v = opscale(v, ks[k]);
      }
      ra[t] = v;
    }
#pragma unroll
    for (int t = 0; t < LPT; ++t) {
      const int e = tid + t * kGemmThreads;
      int cidx, kk;
      if (g.opB == 0) { kk = e % BK; cidx = e / BK; } else { cidx = e % kGemmBN; kk = e / kGemmBN; }
      const int j = j0 + cidx, k = k0 + kk;
      EB v = opzero<EB>();
      if (j < n && k < ke) v = (g.opB == 0) ? B[k + (long long)j * g.ldb] : opconj(B[j + (long long)k * g.ldb]);
      rb[t] = v;
    }
  };
  auto store = [&](int buf) {
#pragma unroll
    for (int t = 0; t < LPT; ++t) {
      const int e = tid + t * kGemmThreads;
      int r, kk;
      if (g.opA == 0) { r = e % kGemmBM; kk = e / kGemmBM; } else { kk = e % BK; r = e / BK; }
      As[buf][kk][r] = ra[t];
    }
#pragma unroll
    for (int t = 0; t < LPT; ++t) {
      const int e = tid + t * kGemmThreads;
      int cidx, kk;
      if (g.opB == 0) { kk = e % BK; cidx = e / BK; } else { cidx = e % kGemmBN; kk = e / kGemmBN; }
      Bs[buf][kk][cidx] = rb[t];
    }
  };
  if (kb < ke) {
    load(kb);
    store(0);
  }
  __syncthreads();
  int buf = 0;
  for (int k0 = kb; k0 < ke; k0 += BK) {
    const bool more = k0 + BK < ke;
    if (more) load(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      EA av[4];
      EB bv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) av[a] = As[buf][kk][tr + 16 * a];
#pragma unroll
      for (int c = 0; c < 4; ++c) bv[c] = Bs[buf][kk][tc + 16 * c];
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int c = 0; c < 4; ++c) opfma(acc[a][c], av[a], bv[c]);
    }
    if (more) store(buf ^ 1);
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int i = i0 + tr + 16 * a, j = j0 + tc + 16 * c;
      if (i >= n || j >= n) continue;
      C v = acc[a][c];
      if (g.outMode == 0) {
        Cm[i + (long long)j * g.ldc] = v;
      } else if (i >= j) {
        if (i == j && g.outMode == 1) v.y = R(0);
        Cm[i + (long long)j * g.ldc] = v;
        if (g.outMode == 1 && i != j) Cm[j + (long long)i * g.ldc] = cconj(v);
      }
    }
}

// ------------------------------------------------------------------------------------
// Householder tridiagonalisation (lower), fused rank-2 update + next mat-vec
// ------------------------------------------------------------------------------------
// Follows the reflector conventions of LAPACK ?hetd2/?larfg: H_i = I - tau v v^H with
// v(0) = 1, H_i^H (alpha; x) = (beta; 0), beta real; A = Q T Q^H, Q = H_0 H_1 ... .
// v(1:) is stored below the subdiagonal of column i of A, tau in tauOut, T in (d, e).
constexpr int kTrdThreads = 1024;   // upper bound (launch bounds); see trd_threads()
// threads per matrix: a matrix of at most 256 (512) rows leaves most of 1024 threads idle
// at barriers, so several CTAs share an SM and hide each other's barrier waits
inline int trd_threads(int Nmax) { return Nmax <= 256 ? 256 : Nmax <= 512 ? 512 : 1024; }

template <typename C, typename R>
__device__ __forceinline__ void householder(C* __restrict__ col, int m, C* __restrict__ v, R* red,
                                            C& tauOut, R& betaOut) {
  // col[0..m): alpha = col[0], x = col[1..m). Produces v[0..m) in smem (v[0] = 1).
  R part = 0;
  for (int r = 1 + threadIdx.x; r < m; r += blockDim.x) part += cabs2(col[r]);
  const R xnorm2 = block_sum(part, red);
  const C alpha = col[0];
  C tau;
  R beta;
  if (xnorm2 == R(0) && alpha.y == R(0)) {
    tau = mk(R(0), R(0));
    beta = alpha.x;
    for (int r = threadIdx.x; r < m; r += blockDim.x) v[r] = mk(r == 0 ? R(1) : R(0), R(0));
  } else {
    const R nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xnorm2);
    beta = (alpha.x >= R(0)) ? -nrm : nrm;
    tau = mk((beta - alpha.x) / beta, -alpha.y / beta);
    // scale = 1 / (alpha - beta)
    const C am = mk(alpha.x - beta, alpha.y);
    const R den = am.x * am.x + am.y * am.y;
    const C sc = mk(am.x / den, -am.y / den);
    for (int r = threadIdx.x; r < m; r += blockDim.x) v[r] = (r == 0) ? mk(R(1), R(0)) : cmul(col[r], sc);
  }
  tauOut = tau;
  betaOut = beta;
}

// Reduce G per-lane values over the 32 lanes of a warp so that column k's total ends in
// the lanes whose id has top log2(G) bits == k (recursive halving: G-1 exchanges instead
// of G full reductions).
template <int G, typename C>
__device__ __forceinline__ C warp_reduce_scatter(C (&v)[G], int lane) {
  constexpr int LG = G == 8 ? 3 : G == 4 ? 2 : G == 2 ? 1 : 0;
#pragma unroll
  for (int s = 0; s < LG; ++s) {
    const int bit = 4 - s;
    const bool hi = (lane >> bit) & 1;
    constexpr int kHalfMax = G / 2;
    const int half = G >> (s + 1);
#pragma unroll
    for (int k = 0; k < kHalfMax; ++k) {
      if (k < half) {
        const C send = hi ? v[k] : v[k + half];
        const C keep = hi ? v[k + half] : v[k];
        C recv;
        recv.x = __shfl_xor_sync(0xffffffffu, send.x, 1 << bit);
        recv.y = __shfl_xor_sync(0xffffffffu, send.y, 1 << bit);
        v[k] = keep + recv;
      }
    }
  }
  C r = v[0];
#pragma unroll
  for (int o = 1; o < (32 >> LG); o <<= 1) {
    r.x += __shfl_xor_sync(0xffffffffu, r.x, o);
    r.y += __shfl_xor_sync(0xffffffffu, r.y, o);
  }
  return r;
}

// off-diagonal tile of 32 rows x 4*NG columns with all rows valid: fully unrolled, no
// predicates. p: this lane's row at the tile's first column; vU, wU, x, y: based at the
// tile's first column.
template <bool UPD, int NG, bool PART>
__device__ __forceinline__ void trd_tile_full(float2* __restrict__ p, long long ld, const float2* __restrict__ vU,
                                              const float2* __restrict__ wU, const float2* __restrict__ x,
                                              float2 vr, float2 wr, float2 xr, float2& ry,
                                              float2* __restrict__ y, int lane, bool rv) {
  // register slot u of a group holds column 4 g + (u ^ q), q = lane >> 3: the columns each
  // lane keeps in the reduce-scatter below are then always slots 0 and 1 (no selects)
  const int q = lane >> 3;
  const float2 z2 = make_float2(0.f, 0.f);
  float2 an[4];
  float2* pn[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    pn[u] = p + (u ^ q) * ld;
    an[u] = (!PART || rv) ? *pn[u] : z2;
  }
  const long long ld4 = 4 * ld;
#pragma unroll
  for (int g = 0; g < NG; ++g) {
    float2 a[4];
    float2* pa[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) { a[u] = an[u]; pa[u] = pn[u]; }
    if (g < NG - 1) {
#pragma unroll
      for (int u = 0; u < 4; ++u) { pn[u] = pa[u] + ld4; an[u] = (!PART || rv) ? *pn[u] : z2; }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int c = 4 * g + (u ^ q);
      if (UPD) {
        const float2 vc = vU[c], wc = wU[c];
        float ax = a[u].x, ay = a[u].y;
        ax = fmaf(-vr.x, wc.x, ax); ax = fmaf(-vr.y, wc.y, ax); ax = fmaf(-wr.x, vc.x, ax); ax = fmaf(-wr.y, vc.y, ax);
        ay = fmaf(-vr.y, wc.x, ay); ay = fmaf(vr.x, wc.y, ay); ay = fmaf(-wr.y, vc.x, ay); ay = fmaf(wr.x, vc.y, ay);
        a[u] = make_float2(ax, ay);
        if (!PART || rv) *pa[u] = a[u];
      }
      const float2 xc = x[c];
      ry.x = fmaf(a[u].x, xc.x, fmaf(-a[u].y, xc.y, ry.x));
      ry.y = fmaf(a[u].x, xc.y, fmaf(a[u].y, xc.x, ry.y));
      a[u] = make_float2(fmaf(a[u].y, xr.y, a[u].x * xr.x), fmaf(-a[u].y, xr.x, a[u].x * xr.y));
    }
    // lanes with bit 4 clear keep columns 0,1 of the group, the others 2,3; then bit 3
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      a[u].x += __shfl_xor_sync(0xffffffffu, a[u + 2].x, 16);
      a[u].y += __shfl_xor_sync(0xffffffffu, a[u + 2].y, 16);
    }
    a[0].x += __shfl_xor_sync(0xffffffffu, a[1].x, 8);
    a[0].y += __shfl_xor_sync(0xffffffffu, a[1].y, 8);
    float2 s = a[0];
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) {
      s.x += __shfl_xor_sync(0xffffffffu, s.x, o);
      s.y += __shfl_xor_sync(0xffffffffu, s.y, o);
    }
    if ((lane & 7) == 0) {
      atomicAdd(&y[4 * g + (lane >> 3)].x, s.x);
      atomicAdd(&y[4 * g + (lane >> 3)].y, s.y);
    }
  }
}

// One pass over the lower triangle of the mm x mm Hermitian block A0 (column-major, ld):
// optionally the rank-2 update A -= vU wU^H + wU vU^H (UPD), and y += A x with the upper
// triangle taken as the conjugate transpose of the lower one. Work unit: 32 rows x 16
// columns per warp (units dealt round-robin), lanes over rows; row sums stay in a
// register, column sums are reduced across lanes G columns at a time; y (shared) is
// accumulated with shared-memory atomics. In single precision the units strictly below
// the diagonal with all rows inside the block (most of them) take the unrolled,
// predicate-free trd_tile_full; diagonal and edge units take the general loop.
template <typename C, typename R, bool UPD>
__device__ __forceinline__ void trd_lower_pass(C* __restrict__ A0, int ld, int mm, const C* __restrict__ vU,
                                               const C* __restrict__ wU, const C* __restrict__ x,
                                               C* __restrict__ y) {
  constexpr int G = sizeof(C) == 8 ? 4 : 2;  // loads in flight per lane within 64 registers
  constexpr int LG = G == 8 ? 3 : G == 4 ? 2 : 1;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int nT = (mm + 31) >> 5;
  constexpr int TC = 16, PR = 2;   // work unit: 32 rows x TC columns; row tile I holds PR (I + 1) units
  const int nTiles = PR * nT * (nT + 1) / 2;
  const C zero = mk(R(0), R(0));
  for (int t = warp; t < nTiles; t += nwarp) {
    int I = (int)((sqrtf(8.0f * (float)(t / PR) + 1.0f) - 1.0f) * 0.5f);
    while (PR * (I + 1) * (I + 2) / 2 <= t) ++I;
    while (PR * I * (I + 1) / 2 > t) --I;
    const int J = t - PR * I * (I + 1) / 2;
    const int r = I * 32 + lane;
    const bool rv = r < mm;
    if constexpr (sizeof(C) == 8) {
      if (J * TC + TC <= I * 32) {
        const C xr = rv ? x[r] : zero;
        const C vr = (UPD && rv) ? vU[r] : zero, wr = (UPD && rv) ? wU[r] : zero;
        C ry = zero;
        C* pr = A0 + (rv ? r : 0) + (long long)J * TC * ld;
        if (I * 32 + 32 <= mm)
          trd_tile_full<UPD, TC / 4, false>(pr, ld, UPD ? vU + J * TC : nullptr, UPD ? wU + J * TC : nullptr,
                                            x + J * TC, vr, wr, xr, ry, y + J * TC, lane, true);
        else
          trd_tile_full<UPD, TC / 4, true>(pr, ld, UPD ? vU + J * TC : nullptr, UPD ? wU + J * TC : nullptr,
                                           x + J * TC, vr, wr, xr, ry, y + J * TC, lane, rv);
        if (rv) {
          atomicAdd(&y[r].x, ry.x);
          atomicAdd(&y[r].y, ry.y);
        }

        continue;
      }
    }
    C vr = zero, wr = zero, xr = zero;
    if (rv) {
      xr = x[r];
      if (UPD) { vr = vU[r]; wr = wU[r]; }
    }
    C ry = zero;
    C* rowp = A0 + (rv ? r : 0);
    const int cEnd = min(mm, J * TC + TC);
    // loads of the next G columns are issued before the current ones are used
    C an[G];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int c = J * TC + u;
      an[u] = (rv && c < mm && c <= r) ? rowp[(long long)c * ld] : zero;
    }
    for (int c0 = J * TC; c0 < cEnd; c0 += G) {
      C a[G];
#pragma unroll
      for (int u = 0; u < G; ++u) a[u] = an[u];
      if (c0 + G < cEnd) {
#pragma unroll
        for (int u = 0; u < G; ++u) {
          const int c = c0 + G + u;
          an[u] = (rv && c < mm && c <= r) ? rowp[(long long)c * ld] : zero;
        }
      }
#pragma unroll
      for (int u = 0; u < G; ++u) {
        const int c = c0 + u;
        const bool ok = rv && c < mm && c <= r;
        if (UPD && ok) {
          a[u] = a[u] - cmulc(vr, wU[c]) - cmulc(wr, vU[c]);
          rowp[(long long)c * ld] = a[u];
        }
        const C xc = (c < mm) ? x[c] : zero;
        if (ok) cfma(ry, a[u], xc);
        // a[u] becomes this lane's contribution conj(a) x_r to y_c (strictly lower part)
        C cp = zero;
        if (ok && c < r) cfma_cj(cp, a[u], xr);
        a[u] = cp;
      }
      const C s = warp_reduce_scatter<G>(a, lane);
      const int cc = c0 + (lane >> (5 - LG));
      if ((lane & ((32 >> LG) - 1)) == 0 && cc < mm) {
        atomicAdd(&y[cc].x, s.x);
        atomicAdd(&y[cc].y, s.y);
      }
    }
    if (rv) {
      atomicAdd(&y[r].x, ry.x);
      atomicAdd(&y[r].y, ry.y);
    }
  }
}

// shared memory of hetrd_kernel: v, w, p, vn, y
constexpr size_t hetrd_smem_bytes(int Nmax, size_t complexBytes) { return 5 * (size_t)Nmax * complexBytes; }

// Unblocked tridiagonalisation of columns i0 .. n-2 of one matrix (A[i0:, i0:] already
// holds every earlier update). Only the lower triangle of A is read or written (the upper
// one is never touched). smem_raw: 5 Nmax elements.
template <typename C, typename R>
__device__ __forceinline__ void hetd2_tail(C* __restrict__ Ab, int n, int Nmax, int i0, double* __restrict__ d,
                                           double* __restrict__ e, C* __restrict__ taus,
                                           unsigned char* __restrict__ smem_raw) {
  C* v = reinterpret_cast<C*>(smem_raw);        // [Nmax] current reflector (relative to row i+1)
  C* w = v + Nmax;                              // [Nmax] w vector
  C* p = w + Nmax;                              // [Nmax] tau*A*v for the next step
  C* vn = p + Nmax;                             // [Nmax] next reflector
  C* y = vn + Nmax;                             // [Nmax] mat-vec accumulator
  __shared__ R red[32];
  __shared__ C s_tau, s_taun;
  __shared__ R s_beta;
  const int tid = threadIdx.x;
  if (n - i0 <= 0) return;
  if (n - i0 == 1) {
    if (tid == 0) { d[i0] = (double)Ab[i0 + (long long)i0 * Nmax].x; }
    return;
  }

  // ---- set-up: reflector of column i0, p = tau A22 v ----
  {
    C t; R be;
    for (int r = tid; r < n; r += blockDim.x) y[r] = mk(R(0), R(0));
    householder<C, R>(Ab + (i0 + 1) + (long long)i0 * Nmax, n - i0 - 1, v, red, t, be);
    if (tid == 0) { s_tau = t; s_beta = be; }
    __syncthreads();
    trd_lower_pass<C, R, false>(Ab + (i0 + 1) + (long long)(i0 + 1) * Nmax, Nmax, n - i0 - 1, nullptr, nullptr, v, y);
    __syncthreads();
    for (int r = tid; r < n - i0 - 1; r += blockDim.x) p[r] = cmul(s_tau, y[r]);
    __syncthreads();
  }

  for (int i = i0; i < n - 1; ++i) {
    const int m = n - i - 1;            // size of A22 = A[i+1:, i+1:]
    const C tau = s_tau;
    const R beta = s_beta;
    // store reflector below the subdiagonal, e, tau, d
    for (int r = 1 + tid; r < m; r += blockDim.x) Ab[(i + 1 + r) + (long long)i * Nmax] = v[r];
    if (tid == 0) {
      e[i] = (double)beta;
      taus[i] = tau;
      d[i] = (double)Ab[i + (long long)i * Nmax].x;
      Ab[(i + 1) + (long long)i * Nmax] = mk(beta, R(0));
    }
    // w = p - 1/2 tau (p^H v) v
    R pr = 0, pi = 0;
    for (int r = tid; r < m; r += blockDim.x) {
      const C pv = cconjmul(p[r], v[r]);
      pr += pv.x;
      pi += pv.y;
    }
    pr = block_sum(pr, red);
    pi = block_sum(pi, red);
    const C pHv = mk(pr, pi);
    const C alph = cscale(cmul(tau, pHv), R(-0.5));
    for (int r = tid; r < m; r += blockDim.x) {
      w[r] = p[r] + cmul(alph, v[r]);
      y[r] = mk(R(0), R(0));
    }
    __syncthreads();
    if (m == 1) {
      // last 1x1 trailing block
      if (tid == 0) {
        C a = Ab[(i + 1) + (long long)(i + 1) * Nmax];
        // a -= v0 conj(w0) + w0 conj(v0)
        a = a - cmulc(v[0], w[0]) - cmulc(w[0], v[0]);
        Ab[(i + 1) + (long long)(i + 1) * Nmax] = a;
        d[i + 1] = (double)a.x;
      }
      break;
    }
    // update first column of A22 (column i+1, rows i+1..n-1)
    C* col = Ab + (i + 1) + (long long)(i + 1) * Nmax;
    for (int r = tid; r < m; r += blockDim.x) {
      C a = col[r];
      a = a - cmulc(v[r], w[0]) - cmulc(w[r], v[0]);
      col[r] = a;
    }
    __syncthreads();
    // next reflector from col[1..m)
    {
      C t; R be;
      householder<C, R>(col + 1, m - 1, vn, red, t, be);
      if (tid == 0) { s_taun = t; s_beta = be; }
    }
    __syncthreads();
    // fused pass over the lower triangle of A33 = A[i+2:, i+2:] (size m-1): rank-2 update
    // with (v[1:], w[1:]) and y = A33_new vn
    const int mm = m - 1;
    trd_lower_pass<C, R, true>(Ab + (i + 2) + (long long)(i + 2) * Nmax, Nmax, mm, v + 1, w + 1, vn, y);
    __syncthreads();
    const C taun = s_taun;
    for (int r = tid; r < mm; r += blockDim.x) {
      p[r] = cmul(taun, y[r]);
      v[r] = vn[r];
    }
    if (tid == 0) s_tau = taun;
    __syncthreads();
  }
}


// order[r] = the matrix of rank r when sorted by size, largest first (ties by index):
// one CTA, rank of each matrix by counting (nb is at most a few thousand)
static __global__ void order_by_size_kernel(const int* __restrict__ nred, int nb, int* __restrict__ order) {
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int nbv = nred[b];
    int rank = 0;
    for (int c = 0; c < nb; ++c) {
      const int nc = nred[c];
      rank += (nc > nbv) || (nc == nbv && c < b);
    }
    order[rank] = b;
  }
}

// Householder tridiagonalisation of every matrix of the batch, unblocked (LAPACK ?hetd2).
template <typename C, typename R>
__global__ void __launch_bounds__(kTrdThreads)
hetrd_kernel(C* __restrict__ A, const int* __restrict__ nred, int Nmax, double* __restrict__ dOut,
             double* __restrict__ eOut, C* __restrict__ tauOut, const int* __restrict__ order = nullptr,
             int /* nBatch: one CTA per matrix here */ = 0) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int b = order ? order[blockIdx.x] : blockIdx.x;
  hetd2_tail<C, R>(A + (long long)b * Nmax * Nmax, nred[b], Nmax, 0, dOut + (long long)b * Nmax,
                   eOut + (long long)b * Nmax, tauOut + (long long)b * Nmax, smem_raw);
}

// sums of two values over the block with one pair of barriers; scratch holds 64 values
template <typename R>
__device__ __forceinline__ void block_sum2(R& a, R& b, R* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) { scratch[wid] = a; scratch[32 + wid] = b; }
  __syncthreads();
  a = warp_sum((lane < nw) ? scratch[lane] : R(0));
  b = warp_sum((lane < nw) ? scratch[32 + lane] : R(0));
}

// Blocked tridiagonalisation (LAPACK ?hetrd with ?latrd panels, lower), single precision.
// Panels of kTrdNB columns: for panel column c the column is brought up to date with the
// panel's earlier reflectors, its reflector v is formed, y = A22 v is a read-only pass over
// the trailing block (stale for this panel), corrected by y -= V (W^H v) + W (V^H v), and
// w = tau y - 1/2 tau (tau y)^H v ... v joins W. After the panel the trailing lower triangle
// takes A -= V W^H + W V^H in one pass (warp per 32 x 32 tile, the row's V and W in
// registers). The last kTrdNX columns use the unblocked hetd2_tail. V and W live in
// shared memory interleaved per reflector, row r: (V[r][q], W[r][q]) for q < kTrdNB.
constexpr int kTrdNB = 8;
constexpr int kTrdNX = 64;
constexpr int kTrdVWS = 2 * kTrdNB + 2;   // float2 row stride of the V/W panel (144 B: 16-byte rows, no bank conflicts)
// shared memory of hetrd_blk_kernel: 5 vectors, the V/W panel, 2 kTrdNB dot products
constexpr size_t hetrd_blk_smem_bytes(int Nmax) {
  return ((5 * (size_t)Nmax * 8 + 15) & ~(size_t)15) + (size_t)Nmax * kTrdVWS * 8 + 2 * kTrdNB * 8;
}

// rank-2 kTrdNB update of the trailing lower triangle rows/cols s0 .. n-1
__device__ __forceinline__ void trd_her2k(float2* __restrict__ Ab, int Nmax, int n, int s0,
                                          const float2* __restrict__ VW) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int mt = n - s0;
  const int nT = (mt + 31) >> 5;
  const int nTiles = nT * (nT + 1) / 2;
  for (int t = warp; t < nTiles; t += nwarp) {
    int I = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    while (I * (I + 1) / 2 > t) --I;
    const int J = t - I * (I + 1) / 2;
    const int r = s0 + I * 32 + lane;
    const bool rv = r < n;
    // this row's (V, W) pairs
    float4 rw[kTrdNB];
    const float4* rp = reinterpret_cast<const float4*>(VW + (long long)(rv ? r : s0) * kTrdVWS);
#pragma unroll
    for (int q = 0; q < kTrdNB; ++q) rw[q] = rp[q];
    const int c0 = s0 + J * 32;
    const int cEnd = min(n, c0 + 32);
    float2* colp = Ab + (rv ? r : s0) + (long long)c0 * Nmax;
#pragma unroll 2
    for (int c = c0; c < cEnd; ++c, colp += Nmax) {
      const float4* cp = reinterpret_cast<const float4*>(VW + (long long)c * kTrdVWS);
      float ax = 0.f, ay = 0.f;
#pragma unroll
      for (int q = 0; q < kTrdNB; ++q) {
        const float4 cq = cp[q];   // (V[c].x, V[c].y, W[c].x, W[c].y)
        // V[r] conj(W[c]) + W[r] conj(V[c])
        ax = fmaf(rw[q].x, cq.z, ax); ax = fmaf(rw[q].y, cq.w, ax);
        ay = fmaf(rw[q].y, cq.z, ay); ay = fmaf(-rw[q].x, cq.w, ay);
        ax = fmaf(rw[q].z, cq.x, ax); ax = fmaf(rw[q].w, cq.y, ax);
        ay = fmaf(rw[q].w, cq.x, ay); ay = fmaf(-rw[q].z, cq.y, ay);
      }
      if (rv && c <= r) {
        float2 a = *colp;
        a.x -= ax;
        a.y -= ay;
        *colp = a;
      }
    }
  }
}

template <typename C, typename R>
__device__ __forceinline__ void hetrd_blk_matrix(C* __restrict__ A, const int* __restrict__ nred, int Nmax,
                                                 double* __restrict__ dOut, double* __restrict__ eOut,
                                                 C* __restrict__ tauOut, int b, unsigned char* smem_raw);

// One CTA per matrix, or (nBatch > gridDim.x) persistent CTAs that take matrices
// blockIdx.x, blockIdx.x + gridDim.x, ... of the size order: fewer matrices in flight keep
// their trailing triangles (the per-column mat-vec passes re-read them) in L2.
template <typename C, typename R>
__global__ void __launch_bounds__(kTrdThreads)
hetrd_blk_kernel(C* __restrict__ A, const int* __restrict__ nred, int Nmax, double* __restrict__ dOut,
                 double* __restrict__ eOut, C* __restrict__ tauOut, const int* __restrict__ order = nullptr,
                 int nBatch = 0) {
  static_assert(sizeof(C) == 8, "single precision");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nb = nBatch > 0 ? nBatch : (int)gridDim.x;
  for (int w = blockIdx.x; w < nb; w += gridDim.x) {
    hetrd_blk_matrix<C, R>(A, nred, Nmax, dOut, eOut, tauOut, order ? order[w] : w, smem_raw);
    __syncthreads();
  }
}

template <typename C, typename R>
__device__ __forceinline__ void hetrd_blk_matrix(C* __restrict__ A, const int* __restrict__ nred, int Nmax,
                                                 double* __restrict__ dOut, double* __restrict__ eOut,
                                                 C* __restrict__ tauOut, int b, unsigned char* smem_raw) {
  const int n = nred[b];
  C* Ab = A + (long long)b * Nmax * Nmax;
  double* d = dOut + (long long)b * Nmax;
  double* e = eOut + (long long)b * Nmax;
  C* taus = tauOut + (long long)b * Nmax;
  C* v = reinterpret_cast<C*>(smem_raw);   // [Nmax] reflector of the current column
  C* y = v + Nmax;                          // [Nmax] mat-vec, then w
  C* VW = reinterpret_cast<C*>(smem_raw + ((5 * (size_t)Nmax * 8 + 15) & ~(size_t)15));  // [Nmax][kTrdVWS]
  C* tq = VW + (long long)Nmax * kTrdVWS;   // [2 kTrdNB] W^H v, then V^H v
  __shared__ R red[64];
  __shared__ C s_tau;
  __shared__ R s_beta;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const int T = blockDim.x;
  const C zero = mk(R(0), R(0));
  int k0 = 0;
  for (; n - k0 > kTrdNX; k0 += kTrdNB) {
    for (int j = 0; j < kTrdNB; ++j) {
      const int c = k0 + j, m = n - c - 1;
      // column c (rows c..n-1) with the panel's earlier reflectors: A -= V W^H + W V^H
      if (j > 0) {
        const C* cw = VW + (long long)c * kTrdVWS;
        for (int r = c + tid; r < n; r += T) {
          const C* rw = VW + (long long)r * kTrdVWS;
          C a = Ab[r + (long long)c * Nmax];
          for (int q = 0; q < j; ++q) a = a - cmulc(rw[2 * q], cw[2 * q + 1]) - cmulc(rw[2 * q + 1], cw[2 * q]);
          if (r == c) a.y = R(0);
          Ab[r + (long long)c * Nmax] = a;
        }
        __syncthreads();
      }
      // reflector from rows c+1..n-1 of column c
      {
        C t; R be;
        householder<C, R>(Ab + (c + 1) + (long long)c * Nmax, m, v, red, t, be);
        if (tid == 0) { s_tau = t; s_beta = be; }
      }
      __syncthreads();
      const C tau = s_tau;
      for (int r = tid; r < m; r += T) {
        const C vr = v[r];
        if (r > 0) Ab[(c + 1 + r) + (long long)c * Nmax] = vr;
        VW[(long long)(c + 1 + r) * kTrdVWS + 2 * j] = vr;
        y[r] = zero;
      }
      if (tid == 0) {
        e[c] = (double)s_beta;
        taus[c] = tau;
        d[c] = (double)Ab[c + (long long)c * Nmax].x;
        Ab[(c + 1) + (long long)c * Nmax] = mk(s_beta, R(0));
      }
      __syncthreads();
      // y = A22 v over the trailing block as stored (read-only pass)
      trd_lower_pass<C, R, false>(Ab + (c + 1) + (long long)(c + 1) * Nmax, Nmax, m, nullptr, nullptr, v, y);
      __syncthreads();
      if (j > 0) {
        // tq[q] = W_q^H v, tq[kTrdNB + q] = V_q^H v (q < j), one warp per dot product
        for (int wq = warp; wq < 2 * j; wq += nwarp) {
          const int q = wq < j ? wq : wq - j;
          const int sel = wq < j ? 1 : 0;   // 1: W column, 0: V column
          C acc = zero;
          for (int r = lane; r < m; r += 32) cfma_cj(acc, VW[(long long)(c + 1 + r) * kTrdVWS + 2 * q + sel], v[r]);
          acc.x = warp_sum(acc.x);
          acc.y = warp_sum(acc.y);
          if (lane == 0) tq[(wq < j ? 0 : kTrdNB) + q] = acc;
        }
        __syncthreads();
      }
      // y -= V (W^H v) + W (V^H v) (j > 0), then w = tau y - 1/2 tau ((tau y)^H v) v -> W
      // column j. Each thread reads and writes only its own rows r of y here (tq and v were
      // published before the last barrier), so one pass does both
      R pr = 0, pi = 0;
      for (int r = tid; r < m; r += T) {
        C s = y[r];
        if (j > 0) {
          const C* rw = VW + (long long)(c + 1 + r) * kTrdVWS;
          for (int q = 0; q < j; ++q) s = s - cmul(rw[2 * q], tq[q]) - cmul(rw[2 * q + 1], tq[kTrdNB + q]);
        }
        const C wv = cmul(tau, s);
        y[r] = wv;
        const C pv = cconjmul(wv, v[r]);
        pr += pv.x;
        pi += pv.y;
      }
      block_sum2(pr, pi, red);
      const C alph = cscale(cmul(tau, mk(pr, pi)), R(-0.5));
      for (int r = tid; r < m; r += T) VW[(long long)(c + 1 + r) * kTrdVWS + 2 * j + 1] = y[r] + cmul(alph, v[r]);
      __syncthreads();
    }
    // trailing block rows/cols k0 + kTrdNB .. n-1
    trd_her2k(Ab, Nmax, n, k0 + kTrdNB, VW);
    __syncthreads();
  }
  hetd2_tail<C, R>(Ab, n, Nmax, k0, d, e, taus, smem_raw);
}

// ------------------------------------------------------------------------------------
// symmetric tridiagonal eigenproblem in FP64: bisection + twisted factorisation
// ------------------------------------------------------------------------------------
constexpr int kTriThreads = 256;

__device__ __forceinline__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e2,
                                           int n, double lam, double pivmin) {
  int cnt = 0;
  double q = d[0] - lam;
  if (fabs(q) < pivmin) q = -pivmin;
  cnt += (q < 0.0);
  for (int k = 1; k < n; ++k) {
    q = (d[k] - lam) - e2[k - 1] / q;
    if (fabs(q) < pivmin) q = -pivmin;
    cnt += (q < 0.0);
  }
  return cnt;
}

// work: [2][n][Nmax] FP64 per matrix (Lp and Um of every eigenvalue, interleaved by
// eigenvalue index so that lanes access consecutive addresses). Z: real eigenvectors,
// row-major Z[k*Nmax + i] = z_i[k], working precision R.
// Eigenvectors are formed only for the eigenvalues in [vecLo, vecHi] (all of them with
// the infinite defaults); their index range [kLo, kHi) goes to krange[2b], krange[2b+1]
// when krange is given, and the other columns of Z are zero. With allValues == 0 only
// the eigenvalues of that range are computed too (two Sturm counts bound it) and the
// other entries of lamOut are zero.
template <typename R>
__global__ void __launch_bounds__(kTriThreads)
tridiag_kernel(const double* __restrict__ dIn, const double* __restrict__ eIn, const int* __restrict__ nred,
               int Nmax, double* __restrict__ lamOut, R* __restrict__ Z, double* __restrict__ work,
               int* __restrict__ status, double vecLo = -INFINITY, double vecHi = INFINITY,
               int* __restrict__ krange = nullptr, int allValues = 1, const int* __restrict__ order = nullptr,
               const int* __restrict__ predK = nullptr, int predMargin = 16, double resTol = -1.0) {
  const int b = order ? order[blockIdx.x] : blockIdx.x;
  const int n = nred[b];
  if (n <= 0) return;
  extern __shared__ double smem_d[];
  double* d = smem_d;            // [Nmax]
  double* e = d + Nmax;          // [Nmax]
  double* e2 = e + Nmax;         // [Nmax]
  double* lam = e2 + Nmax;       // [Nmax]
  __shared__ double red[32];
  const double* db = dIn + (long long)b * Nmax;
  const double* eb = eIn + (long long)b * Nmax;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    d[k] = db[k];
    const double ek = (k < n - 1) ? eb[k] : 0.0;
    e[k] = ek;
    e2[k] = ek * ek;
  }
  __syncthreads();
  // Gershgorin interval and pivmin
  double lo = 1e300, hi = -1e300, emax = 0.0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double r = fabs(e[k]) + (k > 0 ? fabs(e[k - 1]) : 0.0);
    lo = fmin(lo, d[k] - r);
    hi = fmax(hi, d[k] + r);
    emax = fmax(emax, e2[k]);
  }
  lo = block_min(lo, red, 1e300);
  __syncthreads();
  hi = block_max(hi, red, -1e300);
  __syncthreads();
  emax = block_max(emax, red, 0.0);
  const double eps = 2.220446049250313e-16;
  const double tnorm = fmax(fabs(lo), fabs(hi));
  const double pivmin = 2.2250738585072014e-308 * fmax(1.0, emax);
  lo -= 2.0 * eps * tnorm + 4.0 * pivmin;
  hi += 2.0 * eps * tnorm + 4.0 * pivmin;
  // index range of the eigenvalues to compute: all; those in [vecLo, vecHi] (two Sturm
  // counts); or, with a predicted count predK of eigenvalues above vecLo, the largest
  // predK + predMargin (a partial solve sized by the rank predictor, no Sturm count)
  __shared__ int s_vlo, s_vhi;
  if (threadIdx.x == 0) {
    int a = 0, c = n;
    if (predK) {
      a = max(0, n - max(0, predK[b]) - predMargin);
    } else if (!allValues) {
      if (vecLo > lo) a = min(n, sturm_count(d, e2, n, vecLo, pivmin));
      if (vecHi < hi) c = max(a, min(n, sturm_count(d, e2, n, vecHi, pivmin)));
    }
    s_vlo = a;
    s_vhi = c;
  }
  __syncthreads();
  int vLo = s_vlo;
  const int vHi = s_vhi;
  if (predK) {
    for (int i = threadIdx.x; i < vLo; i += blockDim.x) lam[i] = 0.0;
  } else if (!allValues) {
    if (vecLo > lo) lo = vecLo - (2.0 * eps * fabs(vecLo) + 4.0 * pivmin);
    if (vecHi < hi) hi = vecHi + (2.0 * eps * fabs(vecHi) + 4.0 * pivmin);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
      if (i < vLo || i >= vHi) lam[i] = 0.0;
  }
  // bisection for each eigenvalue index
  for (int i = vLo + threadIdx.x; i < vHi; i += blockDim.x) {
    double a = lo, c = hi;
    for (int it = 0; it < 128; ++it) {
      const double mid = 0.5 * (a + c);
      if (mid <= a || mid >= c) break;
      if (c - a <= fmax(2.0 * eps * fmax(fabs(a), fabs(c)), eps * tnorm) + pivmin) break;
      if (sturm_count(d, e2, n, mid, pivmin) > i) c = mid; else a = mid;
    }
    lam[i] = 0.5 * (a + c);
  }
  __syncthreads();
  if (predK && vLo > 0 && lam[vLo] >= vecLo) {
    // the smallest computed (last Ritz) value is still above the threshold, so
    // eigenvalues above it may be missing: fall back to the full solve (all eigenpairs)
    if (threadIdx.x == 0) atomicOr(status + b, (int)kStatusRankFallback);
    for (int i = threadIdx.x; i < vLo; i += blockDim.x) {
      double a = lo, c = hi;
      for (int it = 0; it < 128; ++it) {
        const double mid = 0.5 * (a + c);
        if (mid <= a || mid >= c) break;
        if (c - a <= fmax(2.0 * eps * fmax(fabs(a), fabs(c)), eps * tnorm) + pivmin) break;
        if (sturm_count(d, e2, n, mid, pivmin) > i) c = mid; else a = mid;
      }
      lam[i] = 0.5 * (a + c);
    }
    vLo = 0;
    __syncthreads();
  }
  for (int i = threadIdx.x; i < n; i += blockDim.x) lamOut[(long long)b * Nmax + i] = lam[i];
  // eigenvalue index range of the requested eigenvectors (lam ascending); the partial
  // solve returns the vectors of every value it computed
  __shared__ int s_klo, s_khi;
  if (threadIdx.x == 0) {
    int a = vLo, c = vHi;
    while (!predK && a < c && lam[a] < vecLo) ++a;
    while (!predK && c > a && lam[c - 1] > vecHi) --c;
    s_klo = a;
    s_khi = c;
    if (krange) {
      krange[2 * b] = a;
      krange[2 * b + 1] = c;
    }
  }
  __syncthreads();
  int kLo = s_klo;
  const int kHi = s_khi;

  // twisted factorisation eigenvectors
  double* Lp = work + (long long)b * 2 * Nmax * Nmax;
  double* Um = Lp + (long long)Nmax * Nmax;
  R* Zb = Z + (long long)b * Nmax * Nmax;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    if (i >= kLo && i < kHi) continue;
    for (int k = 0; k < n; ++k) Zb[(long long)k * Nmax + i] = R(0);
  }
  auto twisted = [&](int iBeg, int iEnd) {
  for (int i = iBeg + threadIdx.x; i < iEnd; i += blockDim.x) {
    const double l = lam[i];
    // top-down stationary factorisation T - l = L+ D+ L+^T
    double dp = d[0] - l;
    for (int k = 0; k < n - 1; ++k) {
      if (fabs(dp) < pivmin) dp = -pivmin;
      const double lk = e[k] / dp;
      Lp[(long long)k * Nmax + i] = lk;
      dp = (d[k + 1] - l) - lk * e[k];
    }
    // bottom-up progressive factorisation, twist index r = argmin |gamma|
    // gamma_k = D+_k + D-_k - (d_k - l); D+_k is recomputed from Lp on the way.
    double dm = d[n - 1] - l;
    // D+_{n-1}: recompute forward value for k = n-1
    // we store D+ implicitly: D+_{k+1} = (d_{k+1} - l) - Lp_k e_k
    double best = 1e300;
    int r = n - 1;
    {
      const double dpl = (n > 1) ? ((d[n - 1] - l) - Lp[(long long)(n - 2) * Nmax + i] * e[n - 2]) : (d[0] - l);
      const double gam = dpl + dm - (d[n - 1] - l);
      best = fabs(gam);
      r = n - 1;
    }
    for (int k = n - 2; k >= 0; --k) {
      if (fabs(dm) < pivmin) dm = -pivmin;
      const double uk = e[k] / dm;
      Um[(long long)k * Nmax + i] = uk;
      dm = (d[k] - l) - uk * e[k];
      const double dpk = (k > 0) ? ((d[k] - l) - Lp[(long long)(k - 1) * Nmax + i] * e[k - 1]) : (d[0] - l);
      const double gam = dpk + dm - (d[k] - l);
      if (fabs(gam) < best) {
        best = fabs(gam);
        r = k;
      }
    }
    // z_r = 1; z_k = -Lp_k z_{k+1} (k < r); z_{k+1} = -Um_k z_k (k >= r). Every lane
    // walks the same k (predicated on its own twist index) so accesses stay coalesced.
    // The FP64 values overwrite Lp/Um; the norm is accumulated in FP64.
    double nrm2 = 1.0;
    {
      double z1 = 1.0, z2 = 0.0;  // z_{k+1}, z_{k+2}
      for (int k = n - 2; k >= 0; --k) {
        if (k < r) {
          double zk;
          if (z1 != 0.0) zk = -Lp[(long long)k * Nmax + i] * z1;
          else zk = (e[k] != 0.0) ? -(e[k + 1] / e[k]) * z2 : 0.0;
          nrm2 += zk * zk;
          Lp[(long long)k * Nmax + i] = zk;
          z2 = z1;
          z1 = zk;
        }
      }
    }
    {
      double z1 = 1.0, z2 = 0.0;  // z_k, z_{k-1}
      for (int k = 0; k < n - 1; ++k) {
        if (k >= r) {
          double zn;
          if (z1 != 0.0) zn = -Um[(long long)k * Nmax + i] * z1;
          else zn = (e[k] != 0.0) ? -((k > 0 ? e[k - 1] : 0.0) / e[k]) * z2 : 0.0;
          nrm2 += zn * zn;
          Um[(long long)k * Nmax + i] = zn;  // z_{k+1}
          z2 = z1;
          z1 = zn;
        }
      }
    }
    const double inv = 1.0 / sqrt(nrm2);
    for (int k = 0; k < n; ++k) {
      double zk;
      if (k < r) zk = Lp[(long long)k * Nmax + i];
      else if (k == r) zk = 1.0;
      else zk = Um[(long long)(k - 1) * Nmax + i];
      Zb[(long long)k * Nmax + i] = (R)(zk * inv);
    }
  }
  };
  twisted(kLo, kHi);
  __syncthreads();
  // partial solve: residual check of the computed pairs, |T z - lam z|_inf <= resTol |T|
  // |z|_inf; a larger residual falls back to the full solve (the remaining pairs, which
  // the full solve computes the same way)
  if (predK && resTol >= 0.0 && kLo > 0) {
    __shared__ int s_bad;
    if (threadIdx.x == 0) s_bad = 0;
    __syncthreads();
    for (int i = kLo + threadIdx.x; i < kHi; i += blockDim.x) {
      double res = 0.0, zmax = 0.0;
      for (int k = 0; k < n; ++k) {
        const double zk = (double)Zb[(long long)k * Nmax + i];
        double tz = d[k] * zk;
        if (k > 0) tz += e[k - 1] * (double)Zb[(long long)(k - 1) * Nmax + i];
        if (k < n - 1) tz += e[k] * (double)Zb[(long long)(k + 1) * Nmax + i];
        res = fmax(res, fabs(tz - lam[i] * zk));
        zmax = fmax(zmax, fabs(zk));
      }
      if (!(res <= resTol * tnorm * zmax)) atomicOr(&s_bad, 1);
    }
    __syncthreads();
    if (s_bad) {
      if (threadIdx.x == 0) atomicOr(status + b, (int)(kStatusResidual | kStatusRankFallback));
      for (int i = threadIdx.x; i < kLo; i += blockDim.x) {
        double a = lo, c = hi;
        for (int it = 0; it < 128; ++it) {
          const double mid = 0.5 * (a + c);
          if (mid <= a || mid >= c) break;
          if (c - a <= fmax(2.0 * eps * fmax(fabs(a), fabs(c)), eps * tnorm) + pivmin) break;
          if (sturm_count(d, e2, n, mid, pivmin) > i) c = mid; else a = mid;
        }
        lam[i] = 0.5 * (a + c);
      }
      __syncthreads();
      for (int i = threadIdx.x; i < kLo; i += blockDim.x) lamOut[(long long)b * Nmax + i] = lam[i];
      twisted(0, kLo);
      kLo = 0;
      if (threadIdx.x == 0 && krange) krange[2 * b] = 0;
      __syncthreads();
    }
  }
  // re-orthogonalise tight clusters (relative gap below 1e-10 of |T|): modified
  // Gram-Schmidt inside each cluster, in eigenvalue order.
  const double ctol = 1e-10 * fmax(tnorm, 1e-300);
  __shared__ int s_any;
  if (threadIdx.x == 0) {
    int any = 0;
    for (int i = kLo + 1; i < kHi; ++i) any |= (lam[i] - lam[i - 1] < ctol);
    s_any = any;
  }
  __syncthreads();
  if (!s_any) return;
  if (threadIdx.x == 0) atomicOr(status + b, (int)kStatusClusterFix);
  for (int i = kLo + 1; i < kHi; ++i) {
    if (!(lam[i] - lam[i - 1] < ctol)) continue;
    int j0 = i - 1;
    while (j0 > kLo && lam[j0] - lam[j0 - 1] < ctol) --j0;
    for (int j = j0; j < i; ++j) {
      double part = 0.0;
      for (int k = threadIdx.x; k < n; k += blockDim.x)
        part += (double)Zb[(long long)k * Nmax + i] * (double)Zb[(long long)k * Nmax + j];
      const double dot = block_sum(part, red);
      for (int k = threadIdx.x; k < n; k += blockDim.x)
        Zb[(long long)k * Nmax + i] = (R)((double)Zb[(long long)k * Nmax + i] - dot * (double)Zb[(long long)k * Nmax + j]);
      __syncthreads();
    }
    double part = 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      const double zv = (double)Zb[(long long)k * Nmax + i];
      part += zv * zv;
    }
    const double nr = sqrt(block_sum(part, red));
    const double inv = nr > 0 ? 1.0 / nr : 0.0;
    for (int k = threadIdx.x; k < n; k += blockDim.x)
      Zb[(long long)k * Nmax + i] = (R)((double)Zb[(long long)k * Nmax + i] * inv);
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------
// back-transform Y = Q Z, Q = H_0 ... H_{n-2}; one CTA per (column chunk, matrix)
// ------------------------------------------------------------------------------------
constexpr int kBtThreads = 256;

template <typename C, typename R, int kBtCols>
__global__ void __launch_bounds__(kBtThreads)
backtransform_kernel(const C* __restrict__ A, const C* __restrict__ taus, const R* __restrict__ Z,
                     const int* __restrict__ nred, int Nmax, C* __restrict__ Y, const int* __restrict__ krange,
                const int* __restrict__ order = nullptr) {
  const int b = order ? order[blockIdx.y] : blockIdx.y;
  const int n = nred[b];
  const int c0 = blockIdx.x * kBtCols;
  if (c0 >= n) return;
  // only the eigenvector columns [krange[2b], krange[2b+1]) are needed
  if (krange && (c0 + kBtCols <= krange[2 * b] || c0 >= krange[2 * b + 1])) return;
  const int nc = min(kBtCols, n - c0);
  extern __shared__ unsigned char smem_raw[];
  C* ys = reinterpret_cast<C*>(smem_raw);   // [Nmax][kBtCols]
  C* vs = ys + (long long)Nmax * kBtCols;   // [Nmax]
  C* part = vs + Nmax;                      // [kBtThreads/kBtCols][kBtCols]
  const C* Ab = A + (long long)b * Nmax * Nmax;
  const R* Zb = Z + (long long)b * Nmax * Nmax;
  const C* tb = taus + (long long)b * Nmax;
  const int tid = threadIdx.x;
  for (int e = tid; e < n * kBtCols; e += blockDim.x) {
    const int k = e / kBtCols, c = e % kBtCols;
    ys[e] = mk((c < nc) ? Zb[(long long)k * Nmax + c0 + c] : R(0), R(0));
  }
  __syncthreads();
  const int col = tid % kBtCols, rg = tid / kBtCols, nrg = kBtThreads / kBtCols;
  for (int i = n - 2; i >= 0; --i) {
    const int m = n - i - 1;  // reflector acts on rows i+1 .. n-1
    const C tau = tb[i];
    if (tau.x == R(0) && tau.y == R(0)) continue;
    for (int r = tid; r < m; r += blockDim.x)
      vs[r] = (r == 0) ? mk(R(1), R(0)) : Ab[(i + 1 + r) + (long long)i * Nmax];
    __syncthreads();
    // dot_c = v^H y_c
    C acc = mk(R(0), R(0));
    for (int r = rg; r < m; r += nrg) cfma_cj(acc, vs[r], ys[(i + 1 + r) * kBtCols + col]);
    part[rg * kBtCols + col] = acc;
    __syncthreads();
    if (tid < kBtCols) {
      C s = mk(R(0), R(0));
      for (int g = 0; g < nrg; ++g) s = s + part[g * kBtCols + tid];
      part[tid] = cmul(tau, s);  // tau * v^H y
    }
    __syncthreads();
    const C f = part[col];
    for (int r = rg; r < m; r += nrg) {
      C y = ys[(i + 1 + r) * kBtCols + col];
      y = y - cmul(vs[r], f);
      ys[(i + 1 + r) * kBtCols + col] = y;
    }
    __syncthreads();
  }
  C* Yb = Y + (long long)b * Nmax * Nmax;
  for (int e = tid; e < n * nc; e += blockDim.x) {
    const int k = e % n, c = e / n;
    Yb[k + (long long)(c0 + c) * Nmax] = ys[k * kBtCols + c];
  }
}

// ------------------------------------------------------------------------------------
// blocked back-transform Y = Q Z (compact WY, LAPACK ?larft forward/columnwise + ?larfb)
// ------------------------------------------------------------------------------------
// Reflectors are applied 16 at a time: Q_k = H_i0 ... H_i0+15 = I - V T V^H, so
// Y <- Y - V (T (V^H Y)) for the blocks k = last .. 0. bt_larft_kernel forms T per block
// (one CTA per block and matrix); bt_apply_kernel keeps a 16-column slice of Y in
// registers (thread: one column, every 16th row) for all blocks.
constexpr int kBtNB = 16;             // reflectors per block
constexpr int kBtCB = 16;             // columns of Y per CTA
constexpr int kBtMaxRows = 1024;      // Nmax limit of the register-resident kernel

// element r of reflector i (v(i+1) = 1, stored below the subdiagonal of column i)
template <typename C, typename R>
__device__ __forceinline__ C bt_v(const C* __restrict__ Ab, int Nmax, int i, int r) {
  if (r <= i) return mk(R(0), R(0));
  if (r == i + 1) return mk(R(1), R(0));
  return Ab[r + (long long)i * Nmax];
}

// T of every block of every matrix: Tout[b][k] is 16 x 16 (row-major, upper triangular)
template <typename C, typename R>
__global__ void __launch_bounds__(256)
bt_larft_kernel(const C* __restrict__ A, const C* __restrict__ taus, const int* __restrict__ nred, int Nmax,
                C* __restrict__ Tout, long long tStride) {
  const int b = blockIdx.y, k = blockIdx.x;
  const int n = nred[b];
  const int i0 = k * kBtNB;
  if (i0 >= n - 1) return;
  const int nbk = min(kBtNB, n - 1 - i0);
  const C* Ab = A + (long long)b * Nmax * Nmax;
  const C* tb = taus + (long long)b * Nmax;
  __shared__ C gv[kBtNB][kBtNB];   // gv[l][j] = v_l^H v_j (l < j)
  __shared__ C T[kBtNB][kBtNB];
  __shared__ C t[kBtNB];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int e = tid; e < kBtNB * kBtNB; e += blockDim.x) {
    T[e / kBtNB][e % kBtNB] = mk(R(0), R(0));
    gv[e / kBtNB][e % kBtNB] = mk(R(0), R(0));
  }
  __syncthreads();
  // pairs (l, j), l < j < nbk, one warp per pair; rows from the start of v_j
  for (int pr = warp; pr < nbk * nbk; pr += nwarp) {
    const int l = pr / nbk, j = pr % nbk;
    if (l >= j) continue;
    C acc = mk(R(0), R(0));
    for (int r = i0 + j + 1 + lane; r < n; r += 32)
      cfma_cj(acc, bt_v<C, R>(Ab, Nmax, i0 + l, r), bt_v<C, R>(Ab, Nmax, i0 + j, r));
    acc.x = warp_sum(acc.x);
    acc.y = warp_sum(acc.y);
    if (lane == 0) gv[l][j] = acc;
  }
  __syncthreads();
  for (int j = 0; j < nbk; ++j) {
    const C tauj = tb[i0 + j];
    if (tid < j) t[tid] = cmul(mk(-tauj.x, -tauj.y), gv[tid][j]);
    __syncthreads();
    if (tid < j) {
      C acc = mk(R(0), R(0));
      for (int q = tid; q < j; ++q) cfma(acc, T[tid][q], t[q]);
      T[tid][j] = acc;
    }
    if (tid == 0) T[j][j] = tauj;
    __syncthreads();
  }
  C* To = Tout + (long long)b * tStride + (long long)k * kBtNB * kBtNB;
  for (int e = tid; e < kBtNB * kBtNB; e += blockDim.x) To[e] = T[e / kBtNB][e % kBtNB];
}

// NT threads (256 up to 512 rows, 512 up to 1024 rows). Thread (row group rg = tid / 4,
// column group cg = tid % 4) holds Y rows rg + NT/4 q and columns 4 cg .. 4 cg + 3 of the
// CTA's 16-column slice: every V element loaded from shared memory feeds 4 columns. V^H Y
// partial sums are reduced over the 8 row groups of a warp with shuffles, then over the
// NT/32 warps in shared memory.
constexpr int kBtVS = kBtNB + 2;             // padded row stride of the V block (16-byte aligned rows)
constexpr int kBtJC = 2;                     // reflectors per register chunk

template <typename C, typename R, int KR, int NT, int CB = kBtCB>
__global__ void __launch_bounds__(NT, (sizeof(C) == 8 ? 512 : 256) / NT > 0 ? (sizeof(C) == 8 ? 512 : 256) / NT : 1)
bt_apply_kernel(const C* __restrict__ A, const C* __restrict__ Tin, long long tStride, const R* __restrict__ Z,
                const int* __restrict__ nred, int Nmax, C* __restrict__ Y, const int* __restrict__ krange,
                const int* __restrict__ order = nullptr) {
  const int b = order ? order[blockIdx.y] : blockIdx.y;
  const int n = nred[b];
  const int c0 = blockIdx.x * CB;
  if (c0 >= n) return;
  // only the eigenvector columns [cLo, cHi) are transformed
  const int cLo = krange ? krange[2 * b] : 0, cHi = krange ? krange[2 * b + 1] : n;
  if (c0 + CB <= cLo || c0 >= cHi) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* Vs = reinterpret_cast<C*>(smem_raw);              // [Nmax][kBtVS] block of reflectors (row-major)
  // CGN column groups of 4 columns; RG row groups (the lanes of a warp with the same
  // column group are 32 / CGN of them)
  constexpr int CGN = CB / 4, RG = NT / CGN, NW = NT / 32;
  static_assert(NT >= kBtNB * CB, "one thread per element of W");
  static_assert(CB == 16 || CB == 32, "16 or 32 columns per CTA");
  C* red = Vs + (long long)Nmax * kBtVS;               // [NW warps][16 j][CB c]
  C* Ts = red + NW * kBtNB * CB;                       // [16][16]
  C* Wt = Ts + kBtNB * kBtNB;                          // [16 j][CB c]
  const C* Ab = A + (long long)b * Nmax * Nmax;
  const R* Zb = Z + (long long)b * Nmax * Nmax;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int cg = tid % CGN, rg = tid / CGN;
  C y[KR][4];
#pragma unroll
  for (int q = 0; q < KR; ++q) {
    const int r = rg + RG * q;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int col = c0 + 4 * cg + u;
      // Z (tridiagonal eigenvectors) is row-major: Z(r, col) at r * Nmax + col
      y[q][u] = mk((r < n && col >= cLo && col < cHi) ? Zb[(long long)r * Nmax + col] : R(0), R(0));
    }
  }
  const int nblk = (n - 1 + kBtNB - 1) / kBtNB;
  for (int k = nblk - 1; k >= 0; --k) {
    const int i0 = k * kBtNB;
    const int nbk = min(kBtNB, n - 1 - i0);
    const int m = n - i0 - 1;
    for (int e = tid; e < m * kBtNB; e += blockDim.x) {
      const int r = i0 + 1 + e % m, j = e / m;
      Vs[r * kBtVS + j] = (j < nbk) ? bt_v<C, R>(Ab, Nmax, i0 + j, r) : mk(R(0), R(0));
    }
    const C* Tk = Tin + (long long)b * tStride + (long long)k * kBtNB * kBtNB;
    for (int e = tid; e < kBtNB * kBtNB; e += blockDim.x) {
      const int row = e / kBtNB, cc = e % kBtNB;
      Ts[e] = (row < nbk && cc < nbk) ? Tk[e] : mk(R(0), R(0));
    }
    __syncthreads();
    // W = V^H Y, kBtJC reflectors at a time
#pragma unroll
    for (int jc = 0; jc < kBtNB / kBtJC; ++jc) {
      C w[kBtJC][4];
#pragma unroll
      for (int a = 0; a < kBtJC; ++a)
#pragma unroll
        for (int u = 0; u < 4; ++u) w[a][u] = mk(R(0), R(0));
#pragma unroll
      for (int q = 0; q < KR; ++q) {
        const int r = rg + RG * q;
        if (r > i0 && r < n) {
          C v[kBtJC];
#pragma unroll
          for (int a = 0; a < kBtJC; ++a) v[a] = Vs[r * kBtVS + kBtJC * jc + a];
#pragma unroll
          for (int a = 0; a < kBtJC; ++a)
#pragma unroll
            for (int u = 0; u < 4; ++u) cfma_cj(w[a][u], v[a], y[q][u]);
        }
      }
      // sum over the 8 row groups of the warp (lane bits 2..4)
#pragma unroll
      for (int a = 0; a < kBtJC; ++a)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
          for (int o = CGN; o < 32; o <<= 1) {
            w[a][u].x += __shfl_xor_sync(0xffffffffu, w[a][u].x, o);
            w[a][u].y += __shfl_xor_sync(0xffffffffu, w[a][u].y, o);
          }
        }
      if (lane < CGN) {
#pragma unroll
        for (int a = 0; a < kBtJC; ++a)
#pragma unroll
          for (int u = 0; u < 4; ++u) red[(warp * kBtNB + kBtJC * jc + a) * CB + 4 * cg + u] = w[a][u];
      }
    }
    __syncthreads();
    // W[j][c] over the NW warps, then Wt = T W (thread = (j, c))
    {
      const bool act = tid < kBtNB * CB;
      const int j = (tid / CB) % kBtNB, c = tid % CB;
      C s0 = mk(R(0), R(0));
      if (act) {
#pragma unroll
        for (int g = 0; g < NW; ++g) s0 = s0 + red[(g * kBtNB + j) * CB + c];
      }
      __syncthreads();
      if (act) red[j * CB + c] = s0;
      __syncthreads();
      if (act) {
        C t = mk(R(0), R(0));
        for (int l = j; l < kBtNB; ++l) cfma(t, Ts[j * kBtNB + l], red[l * CB + c]);
        Wt[j * CB + c] = t;
      }
    }
    __syncthreads();
    // Y -= V Wt, kBtJC reflectors at a time
#pragma unroll
    for (int jc = 0; jc < kBtNB / kBtJC; ++jc) {
      C wt[kBtJC][4];
#pragma unroll
      for (int a = 0; a < kBtJC; ++a)
#pragma unroll
        for (int u = 0; u < 4; ++u) wt[a][u] = Wt[(kBtJC * jc + a) * CB + 4 * cg + u];
#pragma unroll
      for (int q = 0; q < KR; ++q) {
        const int r = rg + RG * q;
        if (r > i0 && r < n) {
          C v[kBtJC];
#pragma unroll
          for (int a = 0; a < kBtJC; ++a) v[a] = Vs[r * kBtVS + kBtJC * jc + a];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            C acc = y[q][u];
#pragma unroll
            for (int a = 0; a < kBtJC; ++a) {
              acc.x -= v[a].x * wt[a][u].x - v[a].y * wt[a][u].y;
              acc.y -= v[a].x * wt[a][u].y + v[a].y * wt[a][u].x;
            }
            y[q][u] = acc;
          }
        }
      }
    }
    __syncthreads();
  }
  C* Yb = Y + (long long)b * Nmax * Nmax;
#pragma unroll
  for (int q = 0; q < KR; ++q) {
    const int r = rg + RG * q;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int col = c0 + 4 * cg + u;
      if (r < n && col < n) Yb[r + (long long)col * Nmax] = y[q][u];
    }
  }
}

// shared memory of bt_apply_kernel with nt threads and cb columns per CTA
constexpr size_t bt_apply_smem(int Nmax, size_t complexBytes, int nt, int cb = kBtCB) {
  return ((size_t)Nmax * kBtVS + (nt / 32) * kBtNB * cb + kBtNB * kBtNB + kBtNB * cb) * complexBytes;
}

}  // namespace bippb200
