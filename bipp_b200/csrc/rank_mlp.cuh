// Learned rank predictor: features of the whitened visibility matrix and a small MLP
// (64 -> 128 -> 128 -> 1, ReLU, FP32) that predicts, per time step, the fraction of
// eigenvalues above the energy threshold, so that the tridiagonal stage computes only the
// largest k + margin eigenpairs (a partial solve; tridiag_kernel's predK mode falls back to
// the full solve when the smallest computed value is still above the threshold).
//
// The reference computes every eigenpair with LAPACK ?hegv (src/eigensolver.cpp:188-216)
// and keeps those inside the energy levels afterwards; the predictor has no counterpart
// there. Forward, backward and Adam kernels are hand-written CUDA-core kernels (the layer
// sizes are far below a tensor-core tile): a CTA of 128 threads (one per hidden unit)
// takes a tile of 16 samples; weight gradients of a tile are added with atomics.
#pragma once

#include "common.cuh"

namespace bippb200 {

constexpr int kRankFeatures = 64;
constexpr int kFeatThreads = 512;
constexpr int kMlpH = 128, kMlpTile = 16, kMlpThreads = 128;
// model layout (floats): feature mean and standard deviation (fixed at training time),
// then the trainable parameters W1 [64][128], b1, W2 [128][128], b2, W3 [128], b3
constexpr int kOffMu = 0, kOffSd = kRankFeatures, kOffW1 = 2 * kRankFeatures;
constexpr int kOffB1 = kOffW1 + kRankFeatures * kMlpH, kOffW2 = kOffB1 + kMlpH, kOffB2 = kOffW2 + kMlpH * kMlpH;
constexpr int kOffW3 = kOffB2 + kMlpH, kOffB3 = kOffW3 + kMlpH, kMlpParams = kOffB3 + 1;

// Probe vectors of the trace estimates: Rademacher entries from a hash of (row, probe)
__device__ __forceinline__ float probe_sign(int i, int p) {
  unsigned h = (unsigned)i * 0x9E3779B1u ^ ((unsigned)p * 0x85EBCA77u + 0x165667B1u);
  h ^= h >> 15;
  h *= 0x2C1B3C6Du;
  h ^= h >> 12;
  return (h & 1u) ? 1.f : -1.f;
}

// probes of the trace estimates for matrices of up to nmax rows (their two n x P complex
// work arrays live in shared memory)
inline int rank_probes(int nmax) { return nmax <= 1024 ? 8 : nmax <= 2048 ? 4 : 0; }
// rows of the diagonal / row-norm arrays, even so that the probe arrays after them are
// 8-byte aligned
inline __host__ __device__ int rank_rows(int nmax) { return (nmax + 1) & ~1; }
inline size_t rank_features_smem(int nmax) {
  return 2 * (size_t)rank_rows(nmax) * sizeof(float) + 2 * (size_t)nmax * rank_probes(nmax) * sizeof(float2);
}

// Y = C X for the n x P block X (row-major [n][P] complex in shared memory), C Hermitian
// with its lower triangle at Ab (ld Nmax), in two passes without atomics: a warp per
// column j writes y_j = sum_{i >= j} conj(C_ij) x_i (the column below the diagonal, read
// coalesced and reduced across the warp), then a thread per row i adds
// sum_{j < i} C_ij x_j (the row left of the diagonal; the rows of a warp are consecutive,
// so every column read is coalesced).
template <typename C, int P>
__device__ void herm_block_mv(const C* __restrict__ Ab, int Nmax, int n, const float2* X, float2* Y) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  for (int j = warp; j < n; j += nwarp) {
    float2 acc[P];
#pragma unroll
    for (int p = 0; p < P; ++p) acc[p] = make_float2(0.f, 0.f);
    for (int i = j + lane; i < n; i += 32) {
      const C v = Ab[i + (long long)j * Nmax];
      const float cr = (float)v.x, ci = (i == j) ? 0.f : (float)v.y;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const float2 xi = X[i * P + p];
        acc[p].x += cr * xi.x + ci * xi.y;
        acc[p].y += cr * xi.y - ci * xi.x;
      }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      const float ax = warp_sum(acc[p].x), ay = warp_sum(acc[p].y);
      if (lane == 0) Y[j * P + p] = make_float2(ax, ay);
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    float2 acc[P];
#pragma unroll
    for (int p = 0; p < P; ++p) acc[p] = make_float2(0.f, 0.f);
    for (int j = 0; j < i; ++j) {
      const C v = Ab[i + (long long)j * Nmax];
      const float cr = (float)v.x, ci = (float)v.y;
#pragma unroll
      for (int p = 0; p < P; ++p) {
        const float2 xj = X[j * P + p];
        acc[p].x += cr * xj.x - ci * xj.y;
        acc[p].y += cr * xj.y + ci * xj.x;
      }
    }
#pragma unroll
    for (int p = 0; p < P; ++p) {
      Y[i * P + p].x += acc[p].x;
      Y[i * P + p].y += acc[p].y;
    }
  }
}

// Features of the whitened matrix C = L^-1 S L^-H (lower triangle, ld Nmax) of each step,
// scale-free (divided by the power of the Frobenius norm f = |C|_F that carries C's unit):
//   [0, 32)  the 32 largest |C_ii| (descending)
//   32 log(n) / log(4096); 33 trace C; 34 threshold; 35 fraction of C_ii above the
//   threshold; 36 sum |C_ii|; 37 sum C_ii^2; 38 largest squared row norm; 39 sum of
//   row norms^4; 40 fraction of rows with squared norm above f^2 / n; 41 sum of C_ii above
//   the threshold; 42-45 C_ii at the ranks n/8, n/4, n/2, 3n/4 (descending);
//   46-63 spectral moments t_k = trace C^k, k = 1..6, estimated with P Rademacher probes
//   z (t_k ~ mean z^H C^k z, from Y1 = C Z, Y2 = C Y1, Y3 = C Y2): t3, t4, t5, t6, the
//   effective ranks f^4 / t4 and (f^6 / t6)^(1/2) (both / n), t4^2 / (t6 f^2),
//   t3^2 / (t4 f^2), t5 / (t4 f), their logarithms / log(n), t1 t3 / f^4,
//   t3 / (f t4^(1/2)), t5 / (t4 t6)^(1/2), t2 / f^2 (the probes' own check), and the
//   share of f^2 in the 16 largest rows.
template <typename C, int P>
__global__ void __launch_bounds__(kFeatThreads)
rank_features_kernel(const C* __restrict__ A, int Nmax, const int* __restrict__ nred, double threshold,
                     float* __restrict__ feat) {
  const int b = blockIdx.x;
  const int n = nred[b];
  float* f = feat + (long long)b * kRankFeatures;
  extern __shared__ float fsm[];
  float* dg = fsm;           // [Nmax] diagonal (real)
  float* r2 = fsm + rank_rows(Nmax);   // [Nmax] squared row norms
  float2* Ya = reinterpret_cast<float2*>(fsm + 2 * rank_rows(Nmax));   // [Nmax][P]
  float2* Yb = Ya + (long long)Nmax * P;                     // [Nmax][P]
  __shared__ double red[32];
  __shared__ float top[kRankFeatures];
  __shared__ float rtop[16];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  for (int i = tid; i < kRankFeatures; i += blockDim.x) top[i] = 0.f;
  if (tid < 16) rtop[tid] = 0.f;
  if (n <= 0) {
    for (int i = tid; i < kRankFeatures; i += blockDim.x) f[i] = 0.f;
    return;
  }
  const C* Ab = A + (long long)b * Nmax * Nmax;
  for (int i = tid; i < n; i += blockDim.x) dg[i] = (float)Ab[i + (long long)i * Nmax].x;
  __syncthreads();
  // squared row norms: row j holds its column below the diagonal (conj(C_ij) = C_ji), read
  // by a warp and reduced, and row i holds the entries left of its diagonal, read by a
  // thread per row (consecutive rows, coalesced)
  for (int j = warp; j < n; j += nwarp) {
    float col = 0.f;
    for (int i = j + lane; i < n; i += 32) {
      const C v = Ab[i + (long long)j * Nmax];
      col += (float)v.x * (float)v.x + (float)v.y * (float)v.y;
    }
    col = warp_sum(col);
    if (lane == 0) r2[j] = col;
  }
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) {
    float row = 0.f;
    for (int j = 0; j < i; ++j) {
      const C v = Ab[i + (long long)j * Nmax];
      row += (float)v.x * (float)v.x + (float)v.y * (float)v.y;
    }
    r2[i] += row;
  }
  __syncthreads();
  double sFro = 0, sTr = 0, sAbs = 0, sSq = 0, sR4 = 0, sAbove = 0;
  double cAbove = 0;
  float mR2 = 0.f;
  for (int i = tid; i < n; i += blockDim.x) {
    const double x = dg[i], r = r2[i];
    sFro += r; sTr += x; sAbs += fabs(x); sSq += x * x; sR4 += r * r;
    if (x > threshold) { cAbove += 1; sAbove += x; }
    mR2 = fmaxf(mR2, (float)r);
  }
  const double fro2 = block_sum(sFro, red);
  __syncthreads();
  const double tr = block_sum(sTr, red);
  __syncthreads();
  const double sabs = block_sum(sAbs, red);
  __syncthreads();
  const double ssq = block_sum(sSq, red);
  __syncthreads();
  const double sr4 = block_sum(sR4, red);
  __syncthreads();
  const double cab = block_sum(cAbove, red);
  __syncthreads();
  const double sab = block_sum(sAbove, red);
  __syncthreads();
  const double mr2 = block_max((double)mR2, red, 0.0);
  __syncthreads();
  if (!(fro2 > 0.0)) {
    for (int i = tid; i < kRankFeatures; i += blockDim.x) f[i] = 0.f;
    return;
  }
  const double fro = sqrt(fro2);
  const double cut = fro2 / n;
  double cRows = 0;
  for (int i = tid; i < n; i += blockDim.x) cRows += (r2[i] > cut) ? 1.0 : 0.0;
  const double crow = block_sum(cRows, red);
  __syncthreads();
  // ranks (descending, ties by index): largest |C_ii|, largest row norms, quantiles of C_ii
  const int q1 = n / 8, q2 = n / 4, q3 = n / 2, q4 = (3 * n) / 4;
  for (int i = tid; i < n; i += blockDim.x) {
    const float ai = fabsf(dg[i]), ri = r2[i], si = dg[i];
    int ra = 0, rr = 0, rs = 0;
    for (int j = 0; j < n; ++j) {
      const float aj = fabsf(dg[j]), rj = r2[j], sj = dg[j];
      ra += (aj > ai || (aj == ai && j < i)) ? 1 : 0;
      rr += (rj > ri || (rj == ri && j < i)) ? 1 : 0;
      rs += (sj > si || (sj == si && j < i)) ? 1 : 0;
    }
    if (ra < 32) top[ra] = (float)(ai / fro);
    if (rr < 16) rtop[rr] = ri;
    if (rs == q1) top[42] = (float)(si / fro);
    if (rs == q2) top[43] = (float)(si / fro);
    if (rs == q3) top[44] = (float)(si / fro);
    if (rs == q4) top[45] = (float)(si / fro);
  }
  // spectral moments by probes: Ya = C Z, Yb = C Ya, then Ya = C Yb
  double t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0;
  if constexpr (P > 0) {
    for (int e = tid; e < n * P; e += blockDim.x) Yb[e] = make_float2(probe_sign(e / P, e % P), 0.f);   // Z
    __syncthreads();
    herm_block_mv<C, P>(Ab, Nmax, n, Yb, Ya);
    __syncthreads();
    double a1 = 0, a2 = 0;
    for (int e = tid; e < n * P; e += blockDim.x) {
      const float2 y = Ya[e];
      a1 += (double)probe_sign(e / P, e % P) * y.x;
      a2 += (double)y.x * y.x + (double)y.y * y.y;
    }
    t1 = block_sum(a1, red) / P;
    __syncthreads();
    t2 = block_sum(a2, red) / P;
    __syncthreads();
    herm_block_mv<C, P>(Ab, Nmax, n, Ya, Yb);
    __syncthreads();
    double a3 = 0, a4 = 0;
    for (int e = tid; e < n * P; e += blockDim.x) {
      const float2 x = Ya[e], y = Yb[e];
      a3 += (double)x.x * y.x + (double)x.y * y.y;
      a4 += (double)y.x * y.x + (double)y.y * y.y;
    }
    t3 = block_sum(a3, red) / P;
    __syncthreads();
    t4 = block_sum(a4, red) / P;
    __syncthreads();
    herm_block_mv<C, P>(Ab, Nmax, n, Yb, Ya);
    __syncthreads();
    double a5 = 0, a6 = 0;
    for (int e = tid; e < n * P; e += blockDim.x) {
      const float2 x = Yb[e], y = Ya[e];
      a5 += (double)x.x * y.x + (double)x.y * y.y;
      a6 += (double)y.x * y.x + (double)y.y * y.y;
    }
    t5 = block_sum(a5, red) / P;
    __syncthreads();
    t6 = block_sum(a6, red) / P;
    __syncthreads();
  }
  __syncthreads();
  if (tid == 0) {
    double top16 = 0;
    for (int r = 0; r < 16; ++r) top16 += rtop[r];
    const double ln = log((double)n);
    top[32] = (float)(ln / log(4096.0));
    top[33] = (float)(tr / fro);
    top[34] = (float)(threshold / fro);
    top[35] = (float)(cab / n);
    top[36] = (float)(sabs / fro);
    top[37] = (float)(ssq / fro2);
    top[38] = (float)(mr2 / fro2);
    top[39] = (float)(sr4 / (fro2 * fro2));
    top[40] = (float)(crow / n);
    top[41] = (float)(sab / fro);
    if (P > 0 && t4 > 0 && t6 > 0) {
      const double f3 = fro2 * fro, f4 = fro2 * fro2, f5 = f4 * fro, f6 = f4 * fro2;
      const double er4 = f4 / t4, er6 = sqrt(f6 / t6);
      top[46] = (float)(t3 / f3);
      top[47] = (float)(t4 / f4);
      top[48] = (float)(t5 / f5);
      top[49] = (float)(t6 / f6);
      top[50] = (float)(er4 / n);
      top[51] = (float)(er6 / n);
      top[52] = (float)(t4 * t4 / (t6 * fro2));
      top[53] = (float)(t3 * t3 / (t4 * fro2));
      top[54] = (float)(t5 / (t4 * fro));
      top[55] = (float)(log(fmax(er4, 1e-30)) / ln);
      top[56] = (float)(log(fmax(er6, 1e-30)) / ln);
      top[57] = (float)(t1 * t3 / f4);
      top[58] = (float)(t3 / (fro * sqrt(t4)));
      top[59] = (float)(t5 / sqrt(t4 * t6));
      top[60] = (float)(t2 / fro2);
      top[61] = (float)(t1 / fro);
      top[62] = (float)(er4 / er6);
    }
    top[63] = (float)(top16 / fro2);
  }
  __syncthreads();
  for (int i = tid; i < kRankFeatures; i += blockDim.x) f[i] = top[i];
}

// out[s] = MLP(normalise(X[s])); H1, H2 (optional, [B][128]) keep the activations for
// the backward pass
static __global__ void __launch_bounds__(kMlpThreads)
mlp_forward_kernel(const float* __restrict__ model, const float* __restrict__ X, int B, float* __restrict__ out,
                   float* __restrict__ H1, float* __restrict__ H2) {
  __shared__ float xs[kMlpTile][kRankFeatures];
  __shared__ float h1[kMlpTile][kMlpH];
  __shared__ float part[kMlpThreads / 32][kMlpTile];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int s0 = blockIdx.x * kMlpTile;
  for (int e = t; e < kMlpTile * kRankFeatures; e += kMlpThreads) {
    const int s = e / kRankFeatures, j = e % kRankFeatures;
    const float x = (s0 + s < B) ? X[(long long)(s0 + s) * kRankFeatures + j] : 0.f;
    xs[s][j] = (x - model[kOffMu + j]) / model[kOffSd + j];
  }
  __syncthreads();
  float acc[kMlpTile];
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) acc[s] = model[kOffB1 + t];
  for (int j = 0; j < kRankFeatures; ++j) {
    const float w = model[kOffW1 + j * kMlpH + t];
#pragma unroll
    for (int s = 0; s < kMlpTile; ++s) acc[s] = fmaf(xs[s][j], w, acc[s]);
  }
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) {
    const float a = fmaxf(acc[s], 0.f);
    h1[s][t] = a;
    if (H1 && s0 + s < B) H1[(long long)(s0 + s) * kMlpH + t] = a;
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) acc[s] = model[kOffB2 + t];
  for (int k = 0; k < kMlpH; ++k) {
    const float w = model[kOffW2 + k * kMlpH + t];
#pragma unroll
    for (int s = 0; s < kMlpTile; ++s) acc[s] = fmaf(h1[s][k], w, acc[s]);
  }
  const float w3 = model[kOffW3 + t];
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) {
    const float a = fmaxf(acc[s], 0.f);
    if (H2 && s0 + s < B) H2[(long long)(s0 + s) * kMlpH + t] = a;
    const float p = warp_sum(a * w3);
    if (lane == 0) part[warp][s] = p;
  }
  __syncthreads();
  if (t < kMlpTile && s0 + t < B) {
    float o = model[kOffB3];
#pragma unroll
    for (int w = 0; w < kMlpThreads / 32; ++w) o += part[w][t];
    out[s0 + t] = o;
  }
}

// Gradient of the mean squared error (1/B) sum_s (out_s - Y_s)^2 with respect to the
// trainable parameters, added into grad (model layout; zeroed by the caller), and the
// loss added into loss[*step] (loss[0] without a step counter).
static __global__ void __launch_bounds__(kMlpThreads)
mlp_backward_kernel(const float* __restrict__ model, const float* __restrict__ X, const float* __restrict__ Y, int B,
                    const float* __restrict__ H1, const float* __restrict__ H2, const float* __restrict__ out,
                    float* __restrict__ grad, float* __restrict__ loss, const int* __restrict__ step) {
  __shared__ float xs[kMlpTile][kRankFeatures];
  __shared__ float h1[kMlpTile][kMlpH];
  __shared__ float dz2[kMlpTile][kMlpH];
  __shared__ float g[kMlpTile];
  const int t = threadIdx.x;
  const int s0 = blockIdx.x * kMlpTile;
  for (int e = t; e < kMlpTile * kRankFeatures; e += kMlpThreads) {
    const int s = e / kRankFeatures, j = e % kRankFeatures;
    const float x = (s0 + s < B) ? X[(long long)(s0 + s) * kRankFeatures + j] : 0.f;
    xs[s][j] = (s0 + s < B) ? (x - model[kOffMu + j]) / model[kOffSd + j] : 0.f;
  }
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) h1[s][t] = (s0 + s < B) ? H1[(long long)(s0 + s) * kMlpH + t] : 0.f;
  if (t < 32) {
    float gs = 0.f, ls = 0.f;
    if (t < kMlpTile && s0 + t < B) {
      const float diff = out[s0 + t] - Y[s0 + t];
      gs = 2.f * diff / (float)B;
      ls = diff * diff / (float)B;
    }
    if (t < kMlpTile) g[t] = gs;
    ls = warp_sum(ls);
    if (t == 0) atomicAdd(loss + (step ? *step : 0), ls);
  }
  __syncthreads();
  // output layer
  const float w3 = model[kOffW3 + t];
  float dw3 = 0.f;
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) {
    const float a = (s0 + s < B) ? H2[(long long)(s0 + s) * kMlpH + t] : 0.f;
    dw3 = fmaf(a, g[s], dw3);
    dz2[s][t] = (a > 0.f) ? g[s] * w3 : 0.f;
  }
  atomicAdd(&grad[kOffW3 + t], dw3);
  if (t == 0) {
    float gb = 0.f;
    for (int s = 0; s < kMlpTile; ++s) gb += g[s];
    atomicAdd(&grad[kOffB3], gb);
  }
  __syncthreads();
  // second layer: dW2[k][t] = sum_s h1[s][k] dz2[s][t]
  float db2 = 0.f;
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) db2 += dz2[s][t];
  atomicAdd(&grad[kOffB2 + t], db2);
  for (int k = 0; k < kMlpH; ++k) {
    float v = 0.f;
#pragma unroll
    for (int s = 0; s < kMlpTile; ++s) v = fmaf(h1[s][k], dz2[s][t], v);
    atomicAdd(&grad[kOffW2 + k * kMlpH + t], v);
  }
  // back through W2 and the first ReLU: dz1[s][t] = [h1 > 0] sum_j W2[t][j] dz2[s][j]
  float dz1[kMlpTile];
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) dz1[s] = 0.f;
  for (int j = 0; j < kMlpH; ++j) {
    const float w = model[kOffW2 + t * kMlpH + j];
#pragma unroll
    for (int s = 0; s < kMlpTile; ++s) dz1[s] = fmaf(w, dz2[s][j], dz1[s]);
  }
  float db1 = 0.f;
#pragma unroll
  for (int s = 0; s < kMlpTile; ++s) {
    dz1[s] = (h1[s][t] > 0.f) ? dz1[s] : 0.f;
    db1 += dz1[s];
  }
  atomicAdd(&grad[kOffB1 + t], db1);
  for (int j = 0; j < kRankFeatures; ++j) {
    float v = 0.f;
#pragma unroll
    for (int s = 0; s < kMlpTile; ++s) v = fmaf(xs[s][j], dz1[s], v);
    atomicAdd(&grad[kOffW1 + j * kMlpH + t], v);
  }
}

// Adam step number *step + 1 on the trainable parameters [kOffW1, kMlpParams) (bias
// corrections 1 - beta^t) on the gradient of the loss plus the L2 penalty (l2 / 2) |W|^2
// of the weights (not the biases); the step counter lives on the device so that one
// training iteration can be captured once in a CUDA graph and replayed
static __global__ void mlp_adam_kernel(float* __restrict__ model, const float* __restrict__ grad, float* __restrict__ m,
                                float* __restrict__ v, float lr, float beta1, float beta2, float eps, float l2,
                                const int* __restrict__ step) {
  const float tt = (float)(*step + 1);
  const float c1 = 1.f - powf(beta1, tt), c2 = 1.f - powf(beta2, tt);
  for (int i = kOffW1 + blockIdx.x * blockDim.x + threadIdx.x; i < kMlpParams; i += gridDim.x * blockDim.x) {
    const bool weight = i < kOffB1 || (i >= kOffW2 && i < kOffB2) || (i >= kOffW3 && i < kOffB3);
    const float gi = grad[i] + (weight ? l2 * model[i] : 0.f);
    const float mi = beta1 * m[i] + (1.f - beta1) * gi;
    const float vi = beta2 * v[i] + (1.f - beta2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    model[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

static __global__ void mlp_step_kernel(int* __restrict__ step) { *step += 1; }

// predicted count of eigenvalues above the threshold: round(fraction * n), in [0, n]
static __global__ void rank_predk_kernel(int nb, const float* __restrict__ frac, const int* __restrict__ nred,
                                  int* __restrict__ predK) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const int n = nred[b];
    const float f = frac[b];
    int k = isfinite(f) ? (int)lrintf(f * (float)n) : n;
    predK[b] = max(0, min(n, k));
  }
}

}  // namespace bippb200
