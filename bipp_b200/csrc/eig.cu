// Host driver of the batched generalized eigensolver and the eigh / eigh_gram /
// gram_matrix / virtual_vis C-ABI entry points.
#include <algorithm>
#include <cmath>
#include <complex>
#include <limits>
#include <vector>

#include "context.hpp"
#include "eig.hpp"
#include "rank_mlp.cuh"
#include "tune.hpp"
#include "eig_kernels.cuh"
#include "gemm_tc.cuh"

namespace bippb200 {

// ---------------------------------------------------------------------------------------
// general-W helpers (naive kernels; the batched path uses W = I)
// ---------------------------------------------------------------------------------------
// Gant[a + a' nAnt] = sinc(2 |p_a - p_a'| / wl) (src/host/gram_matrix.cpp:47-56)
__global__ void gram_antenna_kernel(int nAnt, const double* __restrict__ xyz, int ldxyz, double wl,
                                    double* __restrict__ Gant) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nAnt * nAnt;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % nAnt), j = (int)(e / nAnt);
    double g = 1.0;
    if (i != j) {
      const double dx = xyz[i] - xyz[j], dy = xyz[i + ldxyz] - xyz[j + ldxyz], dz = xyz[i + 2 * ldxyz] - xyz[j + 2 * ldxyz];
      const double x = 2.0 * sqrt(dx * dx + dy * dy + dz * dz) / wl;
      g = (x != 0.0) ? sinpi(x) / (3.14159265358979323846 * x) : 1.0;
    }
    Gant[e] = g;
  }
}

// T[a, r] = sum_a' Gant[a, a'] W[a', idx r]   (nAnt x nred, FP64)
template <typename C>
__global__ void gram_gw_kernel(int nAnt, int nred, const double* __restrict__ Gant, const C* __restrict__ W, int ldw,
                               const int* __restrict__ idx, double2* __restrict__ T) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nAnt * nred;
       e += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(e % nAnt), r = (int)(e / nAnt);
    const int col = idx[r];
    double2 acc = make_double2(0, 0);
    for (int ap = 0; ap < nAnt; ++ap) {
      const C wv = W[ap + (long long)col * ldw];
      const double g = Gant[a + (long long)ap * nAnt];
      acc.x += g * (double)wv.x;
      acc.y += g * (double)wv.y;
    }
    T[e] = acc;
  }
}

// G[r, c] = sum_a conj(W[a, idx r]) T[a, c]  (lower triangle, FP64, ld Nmax)
template <typename C>
__global__ void gram_whgw_kernel(int nAnt, int nred, const C* __restrict__ W, int ldw, const int* __restrict__ idx,
                                 const double2* __restrict__ T, double2* __restrict__ G, int Nmax) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nred * nred;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % nred), c = (int)(e / nred);
    if (r < c) continue;
    const int col = idx[r];
    double2 acc = make_double2(0, 0);
    for (int a = 0; a < nAnt; ++a) {
      const C wv = W[a + (long long)col * ldw];
      const double2 t = T[a + (long long)c * nAnt];
      acc.x += (double)wv.x * t.x + (double)wv.y * t.y;
      acc.y += (double)wv.x * t.y - (double)wv.y * t.x;
    }
    if (r == c) acc.y = 0.0;
    G[r + (long long)c * Nmax] = acc;
  }
}

// out (nAnt x nBeam, ld nAnt): identity W -> rows idx[r] = X[r, :]; general W -> W_red X.
template <typename C>
__global__ void unbeam_kernel(int nAnt, int nBeam, int nred, const C* __restrict__ X, int Nmax,
                              const int* __restrict__ idx, const C* __restrict__ W, int ldw, int identity,
                              C* __restrict__ out) {
  using R = decltype(C{}.x);
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nAnt * nBeam;
       e += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(e % nAnt), c = (int)(e / nAnt);
    C v = mk(R(0), R(0));
    if (c < nred) {
      if (identity) {
        // find r with idx[r] == a (idx ascending): binary search
        int lo = 0, hi = nred;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (idx[mid] < a) lo = mid + 1; else hi = mid;
        }
        if (lo < nred && idx[lo] == a) v = X[lo + (long long)c * Nmax];
      } else {
        for (int r = 0; r < nred; ++r) cfma(v, W[a + (long long)idx[r] * ldw], X[r + (long long)c * Nmax]);
      }
    }
    out[e] = v;
  }
}

__global__ void pad_eigenvalues_kernel(int nBatch, int nBeam, const int* __restrict__ nred, const double* __restrict__ lam,
                                       int Nmax, double* __restrict__ out) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nBatch * nBeam;
       e += (long long)gridDim.x * blockDim.x) {
    const int b = (int)(e / nBeam), c = (int)(e % nBeam);
    out[e] = (c < nred[b]) ? lam[(long long)b * Nmax + c] : 0.0;
  }
}

// events between the kernels of one eigensolver sequence (only when timing is requested)
struct SeqTimer {
  cudaStream_t st;
  double* out;
  cudaEvent_t ev[kEigTimers + 1];
  int last = -1;
  SeqTimer(cudaStream_t s, double* o) : st(s), out(o) {
    if (!out) return;
    for (auto& e : ev) cudaEventCreate(&e);
  }
  // mark the start of stage i (closing the previous one)
  void mark(int i) {
    if (!out) return;
    cudaEventRecord(ev[i], st);
    last = i;
  }
  void finish(const int* order, int n) {
    if (!out) return;
    cudaEventRecord(ev[kEigTimers], st);
    cudaEventSynchronize(ev[kEigTimers]);
    for (int k = 0; k < n; ++k) {
      const int a = order[k];
      const int b = (k + 1 < n) ? order[k + 1] : kEigTimers;
      float ms = 0;
      cudaEventElapsedTime(&ms, ev[a], ev[b]);
      out[a] += ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
  }
};

// ---------------------------------------------------------------------------------------
// EigWork
// ---------------------------------------------------------------------------------------
template <typename T>
void EigWork<T>::reserve(bipp_ctx_s* ctx, int nBatch, int nmax) {
  using C = typename Cplx<T>::type;
  const size_t n2 = (size_t)nmax * nmax;
  if (nBatch <= capBatch && nmax == Nmax) return;
  capBatch = nBatch;
  Nmax = nmax;
  A.alloc(ctx, n2 * sizeof(C) * nBatch);
  G.alloc(ctx, n2 * sizeof(double2) * nBatch);
  W64.alloc(ctx, n2 * sizeof(double2) * nBatch);
  Linv.alloc(ctx, n2 * sizeof(C) * nBatch);
  T1.alloc(ctx, n2 * sizeof(C) * nBatch);
  Z.alloc(ctx, n2 * sizeof(T) * nBatch);
  d.alloc(ctx, (size_t)nmax * sizeof(double) * nBatch);
  e.alloc(ctx, (size_t)nmax * sizeof(double) * nBatch);
  tau.alloc(ctx, (size_t)nmax * sizeof(C) * nBatch);
  krange.alloc(ctx, (size_t)2 * sizeof(int) * nBatch);
  order.alloc(ctx, (size_t)sizeof(int) * nBatch);
}

template <typename T>
void eig_launch(bipp_ctx_s* ctx, const EigLaunch<T>& L, EigWork<T>& w) {
  using C = typename Cplx<T>::type;
  using R = T;
  cudaStream_t st = ctx->stream;
  const int nb = L.nBatch, Nmax = L.Nmax;
  const long long n2 = (long long)Nmax * Nmax;
  C* A = w.A.template get<C>();
  double2* G = w.G.template get<double2>();
  double2* W64 = w.W64.template get<double2>();
  C* Linv = w.Linv.template get<C>();
  C* T1 = w.T1.template get<C>();
  R* Z = w.Z.template get<R>();
  const int* nred = L.nred + L.batchOffset;
  int* krange = w.krange.template get<int>();
  SeqTimer tm(st, L.kernelMs);
  int order[kEigTimers];
  int no = 0;
  auto mark = [&](int i) { tm.mark(i); order[no++] = i; };

  // 1. flags (optional) + compaction (+ Gram for W = I)
  mark(0);
  {
    const size_t smem = 2 * (size_t)Nmax * sizeof(int);
    auto k = prep_kernel<T>;
    smem_optin(k, smem);
    count_launch();
    // W = I: the Gram matrix is real symmetric, stored as FP64 reals (withGram 2)
    k<<<nb, kPrepThreads, smem, st>>>(L.nBeam, L.S, L.sStride, L.lds, L.xyz, L.xyzStride, L.ldxyz, L.wl, L.mode,
                                      L.eps, (L.gram && L.identityW) ? 2 : 0, Nmax, L.idx, L.nred, L.nvis, A, G,
                                      L.status, L.doFlag, 1, L.batchOffset);
    B2_CHECK_LAUNCH();
  }
  if (L.gram && !L.identityW) {
    // general W (single matrix): G = W_red^H Gant W_red
    require(nb == 1, "general beamforming matrices are supported for single eigensolves only");
    DevBuf gant(ctx, (size_t)L.nAnt * L.nAnt * sizeof(double));
    DevBuf tmp(ctx, (size_t)L.nAnt * Nmax * sizeof(double2));
    const int nred0 = L.hostNred;
    count_launch();
    gram_antenna_kernel<<<256, 256, 0, st>>>(L.nAnt, L.xyz, L.ldxyz, L.hostWl, gant.get<double>());
    count_launch();
    gram_gw_kernel<C><<<256, 256, 0, st>>>(L.nAnt, nred0, gant.get<double>(), L.W, L.ldw, L.idx, tmp.get<double2>());
    count_launch();
    gram_whgw_kernel<C><<<256, 256, 0, st>>>(L.nAnt, nred0, L.W, L.ldw, L.idx, tmp.get<double2>(), G, Nmax);
    B2_CHECK_LAUNCH();
  }
  // per-matrix kernels take the matrices largest first, so that their last wave holds
  // the smallest ones
  int* sizeOrder = w.order.template get<int>();
  count_launch();
  order_by_size_kernel<<<1, 1024, 0, st>>>(nred, nb, sizeOrder);
  B2_CHECK_LAUNCH();
  const int tiles = (Nmax + kGemmBM - 1) / kGemmBM;
  const bool realG = L.gram && L.identityW;
  if (L.gram) {
    mark(1);
    if (realG) {
      auto k = cholesky_kernel<double>;
      smem_optin(k, chol_smem<double>());
      count_launch();
      k<<<nb, kCholThreads, chol_smem<double>(), st>>>(reinterpret_cast<double*>(G), nred, Nmax,
                                                        L.status + L.batchOffset, sizeOrder);
    } else {
      auto k = cholesky_kernel<double2>;
      smem_optin(k, kCholSmem);
      count_launch();
      k<<<nb, kCholThreads, kCholSmem, st>>>(G, nred, Nmax, L.status + L.batchOffset, sizeOrder);
    }
    B2_CHECK_LAUNCH();
    mark(2);
    if (realG) {
      auto k = trinv_kernel<double, R>;
      smem_optin(k, trinv_smem<double>());
      count_launch();
      k<<<nb, 256, trinv_smem<double>(), st>>>(reinterpret_cast<const double*>(G), reinterpret_cast<double*>(W64),
                                               reinterpret_cast<R*>(Linv), nred, Nmax, sizeOrder);
    } else {
      auto k = trinv_kernel<double2, C>;
      smem_optin(k, kTrinvSmem);
      count_launch();
      k<<<nb, 256, kTrinvSmem, st>>>(G, W64, Linv, nred, Nmax, sizeOrder);
    }
    B2_CHECK_LAUNCH();
    // T1 = Linv * A (Linv real for W = I)
    mark(3);
    GemmArgs<C> g1{};
    g1.A = Linv; g1.strideA = n2; g1.lda = Nmax; g1.opA = 0;
    g1.B = A; g1.strideB = n2; g1.ldb = Nmax; g1.opB = 0;
    g1.Cm = T1; g1.strideC = n2; g1.ldc = Nmax;
    g1.n = nred; g1.triA = 1; g1.triB = 0; g1.outMode = 0; g1.levels = 1;
    // single precision with a real Gram matrix: both products on the tensor cores
    // (C = L^-1 (L^-1 S)^H, Hermitian); otherwise the FP32/FP64 SIMT GEMM
    const bool tcReduce = realG && sizeof(C) == 8;
    count_launch();
    if (tcReduce) {
      if constexpr (sizeof(C) == 8) {
        TgArgs t{};
        t.L = reinterpret_cast<const float*>(Linv); t.strideL = n2; t.ldl = Nmax;
        t.B = A; t.strideB = n2; t.ldb = Nmax; t.opB = 0;
        t.C = T1; t.strideC = n2; t.ldc = Nmax;
        t.n = nred; t.lowerOnly = 0; t.status = L.status + L.batchOffset;
        const dim3 tg((Nmax + kTgM - 1) / kTgM, (Nmax + kTgNC - 1) / kTgNC, nb);
        smem_optin(gemm_tc_kernel, kTgSmem);
        gemm_tc_kernel<<<tg, kTgThreads, kTgSmem, st>>>(t);
      }
    } else if (realG) {
      gemm_kernel<C, R, R, C><<<dim3(tiles, tiles, nb), kGemmThreads, 0, st>>>(g1);
    } else {
      gemm_kernel<C, R><<<dim3(tiles, tiles, nb), kGemmThreads, 0, st>>>(g1);
    }
    B2_CHECK_LAUNCH();
    // A = T1 * Linv^H (Hermitian: lower tiles + mirror)
    GemmArgs<C> g2{};
    g2.A = T1; g2.strideA = n2; g2.lda = Nmax; g2.opA = 0;
    g2.B = Linv; g2.strideB = n2; g2.ldb = Nmax; g2.opB = 1;
    g2.Cm = A; g2.strideC = n2; g2.ldc = Nmax;
    g2.n = nred; g2.triA = 0; g2.triB = 1; g2.outMode = 1; g2.levels = 1;
    count_launch();
    if (tcReduce) {
      if constexpr (sizeof(C) == 8) {
        // only the lower triangle of the reduced matrix is read afterwards
        TgArgs t{};
        t.L = reinterpret_cast<const float*>(Linv); t.strideL = n2; t.ldl = Nmax;
        t.B = T1; t.strideB = n2; t.ldb = Nmax; t.opB = 1;
        t.C = A; t.strideC = n2; t.ldc = Nmax;
        t.n = nred; t.lowerOnly = 1; t.status = L.status + L.batchOffset;
        const dim3 tg((Nmax + kTgM - 1) / kTgM, (Nmax + kTgNC - 1) / kTgNC, nb);
        gemm_tc_kernel<<<tg, kTgThreads, kTgSmem, st>>>(t);
      }
    } else if (realG) {
      gemm_kernel<C, R, C, R><<<dim3(tiles, tiles, nb), kGemmThreads, 0, st>>>(g2);
    } else {
      gemm_kernel<C, R><<<dim3(tiles, tiles, nb), kGemmThreads, 0, st>>>(g2);
    }
    B2_CHECK_LAUNCH();
  }
  // rank predictor: features of the whitened matrix, MLP, predicted counts
  if (L.features) {
    const size_t smem = rank_features_smem(Nmax);
    const int np = rank_probes(Nmax);
    auto k = np == 8 ? rank_features_kernel<C, 8> : np == 4 ? rank_features_kernel<C, 4> : rank_features_kernel<C, 0>;
    smem_optin(k, smem);
    count_launch();
    k<<<nb, kFeatThreads, smem, st>>>(A, Nmax, nred, L.featThreshold, L.features);
    B2_CHECK_LAUNCH();
    if (L.mlpModel) {
      count_launch();
      mlp_forward_kernel<<<(nb + kMlpTile - 1) / kMlpTile, kMlpThreads, 0, st>>>(L.mlpModel, L.features, nb,
                                                                               L.mlpOut, nullptr, nullptr);
      count_launch();
      rank_predk_kernel<<<(nb + 255) / 256, 256, 0, st>>>(nb, L.mlpOut, nred, L.predK);
      B2_CHECK_LAUNCH();
    }
  }
  // 3. tridiagonalisation
  mark(4);
  {
    // single precision: blocked panels while the V/W panel fits in shared memory
    bool blocked = false;
    if constexpr (sizeof(C) == 8) blocked = hetrd_blk_smem_bytes(Nmax) <= ctx->maxSmemOptin;
    const size_t smem = blocked ? hetrd_blk_smem_bytes(Nmax) : hetrd_smem_bytes(Nmax, sizeof(C));
    auto k = hetrd_kernel<C, R>;
    if constexpr (sizeof(C) == 8) {
      if (blocked) k = hetrd_blk_kernel<C, R>;
    }
    smem_optin(k, smem);
    count_launch();
    // threads per matrix: by size, unless the tuning table fixes them; the blocked kernel
    // may run as fewer persistent CTAs (a percentage of the SM count)
    const int tt = tuned("hetrd.threads");
    const int pct = blocked ? tuned("hetrd.ctas_pct") : 0;
    const int grid = pct > 0 ? std::max(1, std::min(nb, pct * ctx->smCount / 100)) : nb;
    k<<<grid, tt > 0 ? tt : trd_threads(Nmax), smem, st>>>(A, nred, Nmax, w.d.template get<double>(),
                                                          w.e.template get<double>(), w.tau.template get<C>(),
                                                          sizeOrder, nb);
    B2_CHECK_LAUNCH();
  }
  // 4. tridiagonal eigenpairs (FP64); workspace aliases W64 (free after trinv)
  mark(5);
  {
    const size_t smem = 4 * (size_t)Nmax * sizeof(double);
    auto k = tridiag_kernel<R>;
    smem_optin(k, smem);
    count_launch();
    // threads per matrix (tunable): by default 128 when only the eigenpairs of a range are
    // computed (one lane per eigenvalue leaves most of 256 idle, and 128-thread CTAs put
    // twice the matrices on an SM), 256 for every eigenpair
    const int tt = tuned("tridiag.threads");
    const int triThreads = tt > 0 ? tt : (L.allValues ? kTriThreads : kTriThreads / 2);
    k<<<nb, triThreads, smem, st>>>(w.d.template get<double>(), w.e.template get<double>(), nred, Nmax,
                                     L.lam + (long long)L.batchOffset * Nmax, Z, reinterpret_cast<double*>(W64),
                                     L.status + L.batchOffset, L.vecLo, L.vecHi, krange, L.allValues, sizeOrder,
                                     L.mlpModel ? L.predK : nullptr, L.predMargin, L.resTol);
    B2_CHECK_LAUNCH();
  }
  // 5. back-transform Y = Q Z -> T1
  mark(6);
  if (Nmax <= (sizeof(C) == 8 ? kBtMaxRows : kBtMaxRows / 2)) {
    // blocked: T of each 16-reflector block into G's storage (free between the triangular
    // inverse and the final GEMM), then one pass over Y per 16-column slice
    C* Tblk = reinterpret_cast<C*>(G);
    const long long tStride = n2 * (long long)(sizeof(double2) / sizeof(C));
    const int nblk = (Nmax - 1 + kBtNB - 1) / kBtNB;
    count_launch();
    bt_larft_kernel<C, R><<<dim3(std::max(1, nblk), nb), 256, 0, st>>>(A, w.tau.template get<C>(), nred, Nmax, Tblk,
                                                                       tStride);
    B2_CHECK_LAUNCH();
#define B2_BT(KR, NT, CB)                                                                    \
  {                                                                                          \
    auto k = bt_apply_kernel<C, R, KR, NT, CB>;                                              \
    const size_t smem = bt_apply_smem(Nmax, sizeof(C), NT, CB);                              \
    smem_optin(k, smem);                                                                     \
    count_launch();                                                                          \
    k<<<dim3((Nmax + CB - 1) / CB, nb), NT, smem, st>>>(A, Tblk, tStride, Z, nred, Nmax, T1, krange, sizeOrder); \
  }
    // up to 512 rows: 16-column slices on 256 threads (64 row groups of 4 column groups), or
    // (tunable) 32-column slices on 512 threads (64 row groups of 8 column groups), which
    // load every reflector block half as often per column; above 512 rows 16-column
    // slices on 512 threads (128 row groups)
    if (Nmax <= 512) {
      const int kr = (Nmax + 63) / 64;
      if (tuned("bt.columns") == 32) {
        if constexpr (sizeof(C) == 8) {
          if (kr <= 2) B2_BT(2, 512, 32) else if (kr <= 4) B2_BT(4, 512, 32) else if (kr <= 6) B2_BT(6, 512, 32) else B2_BT(8, 512, 32)
        } else {
          if (kr <= 2) B2_BT(2, 256, 16) else if (kr <= 4) B2_BT(4, 256, 16) else if (kr <= 6) B2_BT(6, 256, 16) else B2_BT(8, 256, 16)
        }
      } else {
        if (kr <= 2) B2_BT(2, 256, 16) else if (kr <= 4) B2_BT(4, 256, 16) else if (kr <= 6) B2_BT(6, 256, 16) else B2_BT(8, 256, 16)
      }
    } else {
      if constexpr (sizeof(C) == 8) {
        const int kr = (Nmax + 127) / 128;
        if (kr <= 6) B2_BT(6, 512, 16) else B2_BT(8, 512, 16)
      }
    }
#undef B2_BT
    B2_CHECK_LAUNCH();
  } else {
    size_t smem16 = ((size_t)Nmax * 16 + Nmax + kBtThreads) * sizeof(C);
    if (smem16 <= ctx->maxSmemOptin) {
      auto k = backtransform_kernel<C, R, 16>;
      smem_optin(k, smem16);
      count_launch();
      k<<<dim3((Nmax + 15) / 16, nb), kBtThreads, smem16, st>>>(A, w.tau.template get<C>(), Z, nred, Nmax, T1,
                                                                  krange, sizeOrder);
    } else {
      const size_t smem4 = ((size_t)Nmax * 4 + Nmax + kBtThreads) * sizeof(C);
      auto k = backtransform_kernel<C, R, 4>;
      smem_optin(k, smem4);
      count_launch();
      k<<<dim3((Nmax + 3) / 4, nb), kBtThreads, smem4, st>>>(A, w.tau.template get<C>(), Z, nred, Nmax, T1, krange,
                                                              sizeOrder);
    }
    B2_CHECK_LAUNCH();
  }
  // 6. X = Linv^H Y -> X (G storage) ; or X = Y for the standard problem
  if (L.gram) {
    mark(7);
    GemmArgs<C> g3{};
    g3.A = Linv; g3.strideA = n2; g3.lda = Nmax; g3.opA = 1;
    g3.B = T1; g3.strideB = n2; g3.ldb = Nmax; g3.opB = 0;
    g3.Cm = reinterpret_cast<C*>(G); g3.strideC = n2; g3.ldc = Nmax;
    g3.n = nred; g3.triA = 2; g3.triB = 0; g3.outMode = 0; g3.levels = 1; g3.colRange = krange;
    count_launch();
    if (realG)
      gemm_kernel<C, R, R, C><<<dim3(tiles, tiles, nb), kGemmThreads, 0, st>>>(g3);
    else
      gemm_kernel<C, R><<<dim3(tiles, tiles, nb), kGemmThreads, 0, st>>>(g3);
    B2_CHECK_LAUNCH();
  }
  tm.finish(order, no);
}

template <typename T>
typename Cplx<T>::type* EigWork<T>::X(bool gram) {
  using C = typename Cplx<T>::type;
  return gram ? reinterpret_cast<C*>(G.template get<double2>()) : T1.template get<C>();
}

template struct EigWork<float>;
template struct EigWork<double>;
template void eig_launch<float>(bipp_ctx_s*, const EigLaunch<float>&, EigWork<float>&);
template void eig_launch<double>(bipp_ctx_s*, const EigLaunch<double>&, EigWork<double>&);

// ---------------------------------------------------------------------------------------
// single-matrix eigh / eigh_gram (host pointers)
// ---------------------------------------------------------------------------------------
template <typename T>
static void eigh_host(bipp_ctx_s* ctx, bool gram, T wl, size_t nAntenna, size_t nBeam, const void* s, size_t lds,
                      const void* w, size_t ldw, const T* xyz, size_t ldxyz, T* d, void* v, size_t ldv,
                      size_t* nBeamReduced, T* scale) {
  using C = typename Cplx<T>::type;
  using CS = std::complex<T>;
  require(nBeam > 0 && nAntenna > 0, "empty problem");
  require(s && w && d && nBeamReduced && scale, "null pointer", BIPP_INVALID_POINTER_ERROR);
  require(lds >= nBeam && ldw >= nAntenna, "invalid leading dimension");
  require(!gram || (xyz && ldxyz >= nAntenna), "invalid xyz");
  require(!v || ldv >= nAntenna, "invalid ldv");
  require(nBeam <= 4096, "nBeam above the supported maximum of 4096");
  if (sizeof(T) == 8) {
    // complex<double>: the tridiagonalisation keeps 5 rows of nBeam elements and the
    // back-transform 5 nBeam + kBtThreads elements in shared memory
    const size_t cb = sizeof(C), smem = ctx->maxSmemOptin;
    const size_t lim = std::min(smem / (5 * cb), (smem / cb - kBtThreads) / 5);
    if (nBeam > lim)
      throw Error(BIPP_INVALID_PARAMETER_ERROR,
                  "nBeam above the FP64 maximum of " + std::to_string(lim) + " set by this device's shared memory");
  }
  const CS* sp = static_cast<const CS*>(s);
  const CS* wp = static_cast<const CS*>(w);
  // identity beamforming?
  bool identity = (nAntenna == nBeam);
  for (size_t c = 0; identity && c < nBeam; ++c)
    for (size_t r = 0; r < nAntenna; ++r) {
      const CS val = wp[r + c * ldw];
      if (val != CS(r == c ? 1 : 0, 0)) { identity = false; break; }
    }
  const int Nmax = (int)nBeam;
  std::vector<CS> sh(nBeam * nBeam);
  for (size_t c = 0; c < nBeam; ++c)
    for (size_t r = 0; r < nBeam; ++r) sh[r + c * nBeam] = sp[r + c * lds];
  std::vector<double> xyzh(gram ? nAntenna * 3 : 0);
  for (size_t c = 0; gram && c < 3; ++c)
    for (size_t r = 0; r < nAntenna; ++r) xyzh[r + c * nAntenna] = (double)xyz[r + c * ldxyz];
  double wld = (double)wl;

  DevBuf dS(ctx, sh.size() * sizeof(C)), dX(ctx, xyzh.size() * sizeof(double) + 8), dWl(ctx, sizeof(double));
  DevBuf dIdx(ctx, Nmax * sizeof(int)), dNred(ctx, sizeof(int)), dNvis(ctx, sizeof(long long)), dStatus(ctx, sizeof(int));
  DevBuf dLam(ctx, Nmax * sizeof(double));
  DevBuf dW;
  h2d(ctx, dS.get(), sh.data(), sh.size() * sizeof(C));
  if (gram) h2d(ctx, dX.get(), xyzh.data(), xyzh.size() * sizeof(double));
  h2d(ctx, dWl.get(), &wld, sizeof(double));
  dStatus.zero();
  if (!identity || (v && !identity)) {
    std::vector<CS> wh(nAntenna * nBeam);
    for (size_t c = 0; c < nBeam; ++c)
      for (size_t r = 0; r < nAntenna; ++r) wh[r + c * nAntenna] = wp[r + c * ldw];
    dW.alloc(ctx, wh.size() * sizeof(C));
    h2d(ctx, dW.get(), wh.data(), wh.size() * sizeof(C));
  }
  EigWork<T> work;
  work.reserve(ctx, 1, Nmax);
  EigLaunch<T> L{};
  L.nBatch = 1; L.nBeam = (int)nBeam; L.nAnt = (int)nAntenna; L.Nmax = Nmax;
  L.S = dS.get<C>(); L.sStride = (long long)nBeam * nBeam; L.lds = (int)nBeam;
  L.xyz = dX.get<double>(); L.xyzStride = 0; L.ldxyz = (int)nAntenna; L.wl = dWl.get<double>();
  L.hostWl = wld;
  L.mode = gram ? 0 : 1;
  L.eps = std::numeric_limits<T>::epsilon();
  L.gram = gram; L.identityW = identity;
  L.W = dW.get<C>(); L.ldw = (int)nAntenna;
  L.idx = dIdx.get<int>(); L.nred = dNred.get<int>(); L.nvis = dNvis.get<long long>();
  L.status = dStatus.get<int>(); L.lam = dLam.get<double>();
  L.doFlag = 1; L.batchOffset = 0;
  if (gram && !identity) {
    // flags first to know nred for the general-W Gram kernels
    EigLaunch<T> F = L;
    const size_t smem = 2 * (size_t)Nmax * sizeof(int);
    auto k = prep_kernel<T>;
    smem_optin(k, smem);
    count_launch();
    k<<<1, kPrepThreads, smem, ctx->stream>>>(F.nBeam, F.S, F.sStride, F.lds, F.xyz, F.xyzStride, F.ldxyz, F.wl,
                                              F.mode, F.eps, 0, Nmax, F.idx, F.nred, F.nvis,
                                              work.A.template get<C>(), work.G.template get<double2>(), F.status, 1, 0, 0);
    B2_CHECK_LAUNCH();
    int nr = 0;
    d2h(ctx, &nr, dNred.get(), sizeof(int));
    sync(ctx);
    L.hostNred = nr;
    L.doFlag = 0;
  }
  eig_launch<T>(ctx, L, work);
  int nred = 0, status = 0;
  long long nvis = 0;
  d2h(ctx, &nred, dNred.get(), sizeof(int));
  d2h(ctx, &nvis, dNvis.get(), sizeof(long long));
  d2h(ctx, &status, dStatus.get(), sizeof(int));
  std::vector<double> lam(Nmax);
  d2h(ctx, lam.data(), dLam.get(), Nmax * sizeof(double));
  DevBuf dOut;
  if (v) {
    dOut.alloc(ctx, nAntenna * nBeam * sizeof(C));
    count_launch();
    unbeam_kernel<C><<<256, 256, 0, ctx->stream>>>((int)nAntenna, (int)nBeam, nred > 0 ? nred : 0,
                                                   work.X(gram), Nmax, dIdx.get<int>(), dW.get<C>(), (int)nAntenna,
                                                   identity ? 1 : 0, dOut.get<C>());
    B2_CHECK_LAUNCH();
  }
  sync(ctx);
  // nred from the flag pass is authoritative even when nred was 0 (kernels skipped)
  if (status & kStatusTensorTimeout) throw Error(BIPP_GPU_ERROR, "tensor-core MMA wait timed out");
  if (status & kStatusCholeskyNotPD) throw Error(BIPP_EIGENSOLVER_ERROR, "Gram matrix is not positive definite");
  if (status & kStatusNonFinite) throw Error(BIPP_EIGENSOLVER_ERROR, "non-finite visibility in a kept entry of S");
  if (nred == 0) {
    // every row and column flagged: the reference zeroes d and v, then hands LAPACK a
    // 0 x 0 problem with leading dimension 0, which LAPACK rejects (info < 0), and throws
    // EigensolverError (src/eigensolver.cpp:172-173, src/host/lapack_api.hpp:133)
    for (size_t c = 0; c < nBeam; ++c) d[c] = T(0);
    if (v)
      for (size_t c = 0; c < nBeam; ++c)
        for (size_t r = 0; r < nAntenna; ++r) static_cast<CS*>(v)[r + c * ldv] = CS(0, 0);
    throw Error(BIPP_EIGENSOLVER_ERROR, "every row and column of S is flagged (empty eigenproblem)");
  }
  for (size_t c = 0; c < nBeam; ++c) d[c] = (c < (size_t)nred) ? (T)lam[c] : T(0);
  if (v) {
    B2_CUDA(cudaMemcpy2DAsync(v, ldv * sizeof(C), dOut.get(), nAntenna * sizeof(C), nAntenna * sizeof(C), nBeam,
                              cudaMemcpyDeviceToHost, ctx->stream));
    sync(ctx);
  }
  *nBeamReduced = (size_t)nred;
  *scale = nvis ? T(1) / T(nvis) : T(0);
}

// columns of v (nAnt x nAnt) outside the computed eigenvector range [kLo, kHi) of the
// matrix (the ranked solves compute part of the eigenpairs) set to zero
__global__ void zero_outside_range_kernel(int nAnt, const int* __restrict__ krange, float2* __restrict__ v) {
  const int kLo = krange[0], kHi = krange[1];
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nAnt * nAnt;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / nAnt);
    if (c < kLo || c >= kHi) v[e] = make_float2(0.f, 0.f);
  }
}

// batched eigh_gram, W = I; with `ro` (single precision) the ranked forms: the full solve,
// the exact range above a threshold (Sturm counts) or the predicted partial solve
template <typename T>
static void eigh_gram_batched_host(bipp_ctx_s* ctx, size_t nBatch, size_t nAnt, const T* wl, const void* s,
                                   const T* xyz, T* d, void* v, size_t* nBeamReduced, T* scale,
                                   const RankOpts* ro = nullptr) {
  using C = typename Cplx<T>::type;
  require(nBatch > 0 && nAnt > 0, "empty problem");
  require(s && xyz && wl && d && nBeamReduced && scale, "null pointer", BIPP_INVALID_POINTER_ERROR);
  require(nAnt <= 4096, "nAntenna above the supported maximum of 4096");
  if (sizeof(T) == 8) {
    // as eigh_host: FP64 rows of the tridiagonalisation and back-transform in shared memory
    const size_t cb = sizeof(C), smem = ctx->maxSmemOptin;
    const size_t lim = std::min(smem / (5 * cb), (smem / cb - kBtThreads) / 5);
    if (nAnt > lim)
      throw Error(BIPP_INVALID_PARAMETER_ERROR,
                  "nAntenna above the FP64 maximum of " + std::to_string(lim) + " set by this device's shared memory");
  }
  const int Nmax = (int)nAnt;
  const size_t chunk = std::min<size_t>(nBatch, 256);
  const size_t n2 = nAnt * nAnt;
  std::vector<double> xyzh(nBatch * nAnt * 3), wlh(nBatch);
  for (size_t i = 0; i < xyzh.size(); ++i) xyzh[i] = xyz[i];
  for (size_t i = 0; i < nBatch; ++i) wlh[i] = wl[i];
  DevBuf dS(ctx, chunk * n2 * sizeof(C)), dX(ctx, xyzh.size() * sizeof(double)), dWl(ctx, nBatch * sizeof(double));
  DevBuf dIdx(ctx, nBatch * Nmax * sizeof(int)), dNred(ctx, nBatch * sizeof(int)), dNvis(ctx, nBatch * sizeof(long long));
  DevBuf dStatus(ctx, nBatch * sizeof(int)), dLam(ctx, nBatch * Nmax * sizeof(double)), dLamPad(ctx, chunk * nAnt * sizeof(double));
  DevBuf dV(ctx, chunk * n2 * sizeof(C));
  h2d(ctx, dX.get(), xyzh.data(), xyzh.size() * sizeof(double));
  h2d(ctx, dWl.get(), wlh.data(), nBatch * sizeof(double));
  dStatus.zero();
  EigWork<T> work;
  work.reserve(ctx, (int)chunk, Nmax);
  DevBuf dModel, dFeat, dOut, dPredK;
  if (ro) {
    require(ro->mode >= 0 && ro->mode <= 2, "unknown rank mode");
    require(ro->mode != 2 || ro->modelHost, "the predicted partial solve needs a model", BIPP_INVALID_POINTER_ERROR);
    require(ro->margin >= 0, "negative margin");
    if (ro->mode == 2) {
      dModel.alloc(ctx, kMlpParams * sizeof(float));
      h2d(ctx, dModel.get(), ro->modelHost, kMlpParams * sizeof(float));
      dOut.alloc(ctx, chunk * sizeof(float));
      dPredK.alloc(ctx, chunk * sizeof(int));
    }
    if (ro->mode == 2 || ro->features) dFeat.alloc(ctx, chunk * kRankFeatures * sizeof(float));
  }
  std::vector<int> kr(2 * chunk);
  cudaEvent_t evA = nullptr, evB = nullptr;
  if (ro && ro->ms) {
    B2_CUDA(cudaEventCreate(&evA));
    B2_CUDA(cudaEventCreate(&evB));
    *ro->ms = 0.0;
  }
  std::vector<int> nredh(nBatch);
  std::vector<long long> nvish(nBatch);
  std::vector<int> stat(nBatch);
  std::vector<double> lamh(chunk * nAnt);
  for (size_t b0 = 0; b0 < nBatch; b0 += chunk) {
    const size_t nb = std::min(chunk, nBatch - b0);
    h2d(ctx, dS.get(), static_cast<const char*>(s) + b0 * n2 * sizeof(C), nb * n2 * sizeof(C));
    EigLaunch<T> L{};
    L.nBatch = (int)nb; L.nBeam = (int)nAnt; L.nAnt = (int)nAnt; L.Nmax = Nmax;
    L.S = dS.get<C>(); L.sStride = (long long)n2; L.lds = (int)nAnt;
    L.xyz = dX.get<double>(); L.xyzStride = (long long)nAnt * 3; L.ldxyz = (int)nAnt; L.wl = dWl.get<double>();
    L.mode = 0; L.eps = std::numeric_limits<T>::epsilon();
    L.gram = true; L.identityW = true;
    L.idx = dIdx.get<int>(); L.nred = dNred.get<int>(); L.nvis = dNvis.get<long long>();
    L.status = dStatus.get<int>(); L.lam = dLam.get<double>();
    L.doFlag = 1; L.batchOffset = (int)b0;
    if (ro) {
      if (ro->mode >= 1) {
        L.allValues = 0;
        L.vecLo = ro->threshold;
        L.vecHi = INFINITY;
      }
      if (ro->mode == 2 || ro->features) {
        L.features = dFeat.get<float>();
        L.featThreshold = ro->threshold;
      }
      if (ro->mode == 2) {
        L.mlpModel = dModel.get<float>();
        L.mlpOut = dOut.get<float>();
        L.predK = dPredK.get<int>();
        L.predMargin = ro->margin;
        L.resTol = ro->resTol;
      }
      if (evA) B2_CUDA(cudaEventRecord(evA, ctx->stream));
    }
    eig_launch<T>(ctx, L, work);
    if (ro) {
      if (evB) {
        B2_CUDA(cudaEventRecord(evB, ctx->stream));
        B2_CUDA(cudaEventSynchronize(evB));
        float t = 0.f;
        B2_CUDA(cudaEventElapsedTime(&t, evA, evB));
        *ro->ms += t;
      }
      if (ro->features) d2h(ctx, ro->features + b0 * kRankFeatures, dFeat.get(), nb * kRankFeatures * sizeof(float));
      d2h(ctx, kr.data(), work.krange.get(), 2 * nb * sizeof(int));
    }
    // outputs for this chunk: scatter each matrix's eigenvectors to its kept antenna rows
    std::vector<int> nr(nb);
    d2h(ctx, nr.data(), dNred.get<int>() + b0, nb * sizeof(int));
    sync(ctx);
    for (size_t b = 0; b < nb; ++b) {
      count_launch();
      unbeam_kernel<C><<<128, 256, 0, ctx->stream>>>((int)nAnt, (int)nAnt, nr[b],
                                                     work.X(true) + (long long)b * Nmax * Nmax, Nmax,
                                                     dIdx.get<int>() + (b0 + b) * Nmax, nullptr, 0, 1,
                                                     dV.get<C>() + b * n2);
      if constexpr (sizeof(T) == 4) {
        if (ro && ro->mode >= 1) {
          count_launch();
          zero_outside_range_kernel<<<128, 256, 0, ctx->stream>>>((int)nAnt, work.krange.template get<int>() + 2 * b,
                                                                  dV.get<float2>() + b * n2);
        }
      }
    }
    B2_CHECK_LAUNCH();
    count_launch();
    pad_eigenvalues_kernel<<<64, 256, 0, ctx->stream>>>((int)nb, (int)nAnt, dNred.get<int>() + b0,
                                                        dLam.get<double>() + b0 * Nmax, Nmax, dLamPad.get<double>());
    B2_CHECK_LAUNCH();
    d2h(ctx, lamh.data(), dLamPad.get(), nb * nAnt * sizeof(double));
    if (v) d2h(ctx, static_cast<char*>(v) + b0 * n2 * sizeof(C), dV.get(), nb * n2 * sizeof(C));
    sync(ctx);
    for (size_t i = 0; i < nb * nAnt; ++i) d[b0 * nAnt + i] = (T)lamh[i];
    if (ro && ro->kComputed)
      for (size_t b = 0; b < nb; ++b) ro->kComputed[b0 + b] = nr[b] ? kr[2 * b + 1] - kr[2 * b] : 0;
  }
  if (evA) cudaEventDestroy(evA);
  if (evB) cudaEventDestroy(evB);
  d2h(ctx, nredh.data(), dNred.get(), nBatch * sizeof(int));
  d2h(ctx, nvish.data(), dNvis.get(), nBatch * sizeof(long long));
  d2h(ctx, stat.data(), dStatus.get(), nBatch * sizeof(int));
  sync(ctx);
  for (size_t b = 0; b < nBatch; ++b) {
    if (stat[b] & kStatusTensorTimeout) throw Error(BIPP_GPU_ERROR, "tensor-core MMA wait timed out");
    if (stat[b] & kStatusCholeskyNotPD) throw Error(BIPP_EIGENSOLVER_ERROR, "Gram matrix is not positive definite");
    if (stat[b] & kStatusNonFinite) throw Error(BIPP_EIGENSOLVER_ERROR, "non-finite visibility in a kept entry of S");
    if (nredh[b] == 0) throw Error(BIPP_EIGENSOLVER_ERROR, "every row and column of S is flagged (empty eigenproblem)");
    nBeamReduced[b] = (size_t)nredh[b];
    scale[b] = nvish[b] ? T(1) / (T)nvish[b] : T(0);
    if (ro && ro->fallback) ro->fallback[b] = (stat[b] & kStatusRankFallback) ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------------------
// gram_matrix / virtual_vis (host pointers)
// ---------------------------------------------------------------------------------------
template <typename T>
static void gram_host(bipp_ctx_s* ctx, size_t nAnt, size_t nBeam, const void* w, size_t ldw, const T* xyz,
                      size_t ldxyz, T wl, void* g, size_t ldg) {
  using C = typename Cplx<T>::type;
  using CS = std::complex<T>;
  require(w && xyz && g, "null pointer", BIPP_INVALID_POINTER_ERROR);
  require(ldw >= nAnt && ldxyz >= nAnt && ldg >= nBeam, "invalid leading dimension");
  std::vector<double> xyzh(nAnt * 3);
  for (size_t c = 0; c < 3; ++c)
    for (size_t r = 0; r < nAnt; ++r) xyzh[r + c * nAnt] = (double)xyz[r + c * ldxyz];
  std::vector<CS> wh(nAnt * nBeam);
  const CS* wp = static_cast<const CS*>(w);
  for (size_t c = 0; c < nBeam; ++c)
    for (size_t r = 0; r < nAnt; ++r) wh[r + c * nAnt] = wp[r + c * ldw];
  std::vector<int> idx(nBeam);
  for (size_t i = 0; i < nBeam; ++i) idx[i] = (int)i;
  DevBuf dX(ctx, xyzh.size() * sizeof(double)), dW(ctx, wh.size() * sizeof(C)), dIdx(ctx, nBeam * sizeof(int));
  DevBuf gant(ctx, nAnt * nAnt * sizeof(double)), tmp(ctx, nAnt * nBeam * sizeof(double2)),
      dG(ctx, nBeam * nBeam * sizeof(double2));
  h2d(ctx, dX.get(), xyzh.data(), xyzh.size() * sizeof(double));
  h2d(ctx, dW.get(), wh.data(), wh.size() * sizeof(C));
  h2d(ctx, dIdx.get(), idx.data(), idx.size() * sizeof(int));
  count_launch();
  gram_antenna_kernel<<<256, 256, 0, ctx->stream>>>((int)nAnt, dX.get<double>(), (int)nAnt, (double)wl, gant.get<double>());
  count_launch();
  gram_gw_kernel<C><<<256, 256, 0, ctx->stream>>>((int)nAnt, (int)nBeam, gant.get<double>(), dW.get<C>(), (int)nAnt,
                                                  dIdx.get<int>(), tmp.get<double2>());
  dG.zero();
  count_launch();
  gram_whgw_kernel<C><<<256, 256, 0, ctx->stream>>>((int)nAnt, (int)nBeam, dW.get<C>(), (int)nAnt, dIdx.get<int>(),
                                                    tmp.get<double2>(), dG.get<double2>(), (int)nBeam);
  B2_CHECK_LAUNCH();
  std::vector<std::complex<double>> gh(nBeam * nBeam);
  d2h(ctx, gh.data(), dG.get(), gh.size() * sizeof(double2));
  sync(ctx);
  CS* gp = static_cast<CS*>(g);
  for (size_t c = 0; c < nBeam; ++c)
    for (size_t r = 0; r < nBeam; ++r) {
      const std::complex<double> val = (r >= c) ? gh[r + c * nBeam] : std::conj(gh[c + r * nBeam]);
      gp[r + c * ldg] = CS((T)val.real(), (T)val.imag());
    }
}

template <typename T>
static void virtual_vis_host(bipp_ctx_s* ctx, T scale, size_t nAnt, size_t nBeam, const T* d, const void* v, size_t ldv,
                             void* vv) {
  using C = typename Cplx<T>::type;
  require(d && v && vv, "null pointer", BIPP_INVALID_POINTER_ERROR);
  require(ldv >= nAnt, "invalid leading dimension");
  std::vector<T> ks(nBeam);
  for (size_t i = 0; i < nBeam; ++i) ks[i] = scale * d[i];
  DevBuf dV(ctx, nAnt * nBeam * sizeof(C)), dK(ctx, nBeam * sizeof(T)), dVV(ctx, nAnt * nAnt * sizeof(C));
  DevBuf dn(ctx, 3 * sizeof(int));
  B2_CUDA(cudaMemcpy2DAsync(dV.get(), nAnt * sizeof(C), v, ldv * sizeof(C), nAnt * sizeof(C), nBeam,
                            cudaMemcpyHostToDevice, ctx->stream));
  h2d(ctx, dK.get(), ks.data(), nBeam * sizeof(T));
  int hn[3] = {(int)nAnt, 0, (int)nBeam};
  h2d(ctx, dn.get(), hn, sizeof(hn));
  GemmArgs<C> g{};
  g.A = dV.get<C>(); g.lda = (int)nAnt; g.opA = 0;
  g.B = dV.get<C>(); g.ldb = (int)nAnt; g.opB = 1;
  g.Cm = dVV.get<C>(); g.ldc = (int)nAnt;
  g.n = dn.get<int>(); g.outMode = 0; g.levels = 1;
  g.kscale = dK.get(); g.kbeg = dn.get<int>() + 1; g.kend = dn.get<int>() + 2;
  const int tiles = ((int)nAnt + kGemmBM - 1) / kGemmBM;
  count_launch();
  gemm_kernel<C, T><<<dim3(tiles, tiles, 1), kGemmThreads, 0, ctx->stream>>>(g);
  B2_CHECK_LAUNCH();
  d2h(ctx, vv, dVV.get(), nAnt * nAnt * sizeof(C));
  sync(ctx);
}

}  // namespace bippb200

using namespace bippb200;

extern "C" {

BippError bipp_eigh_gram_s(bipp_ctx_t ctx, float wl, size_t nAntenna, size_t nBeam, const void* s, size_t lds,
                           const void* w, size_t ldw, const float* xyz, size_t ldxyz, float* d, void* v, size_t ldv,
                           size_t* nBeamReduced, float* scale) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    eigh_host<float>(ctx, true, wl, nAntenna, nBeam, s, lds, w, ldw, xyz, ldxyz, d, v, ldv, nBeamReduced, scale);
  });
}
BippError bipp_eigh_gram_d(bipp_ctx_t ctx, double wl, size_t nAntenna, size_t nBeam, const void* s, size_t lds,
                           const void* w, size_t ldw, const double* xyz, size_t ldxyz, double* d, void* v, size_t ldv,
                           size_t* nBeamReduced, double* scale) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    eigh_host<double>(ctx, true, wl, nAntenna, nBeam, s, lds, w, ldw, xyz, ldxyz, d, v, ldv, nBeamReduced, scale);
  });
}
BippError bipp_eigh_s(bipp_ctx_t ctx, float wl, size_t nAntenna, size_t nBeam, const void* s, size_t lds, const void* w,
                      size_t ldw, float* d, void* v, size_t ldv, size_t* nBeamReduced, float* scale) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    eigh_host<float>(ctx, false, wl, nAntenna, nBeam, s, lds, w, ldw, nullptr, 0, d, v, ldv, nBeamReduced, scale);
  });
}
BippError bipp_eigh_d(bipp_ctx_t ctx, double wl, size_t nAntenna, size_t nBeam, const void* s, size_t lds, const void* w,
                      size_t ldw, double* d, void* v, size_t ldv, size_t* nBeamReduced, double* scale) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    eigh_host<double>(ctx, false, wl, nAntenna, nBeam, s, lds, w, ldw, nullptr, 0, d, v, ldv, nBeamReduced, scale);
  });
}
BippError bipp_eigh_gram_batched_s(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna, const float* wl, const void* s,
                                   const float* xyz, float* d, void* v, size_t* nBeamReduced, float* scale) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    eigh_gram_batched_host<float>(ctx, nBatch, nAntenna, wl, s, xyz, d, v, nBeamReduced, scale);
  });
}
BippError bipp_eigh_gram_batched_d(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna, const double* wl, const void* s,
                                   const double* xyz, double* d, void* v, size_t* nBeamReduced, double* scale) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    eigh_gram_batched_host<double>(ctx, nBatch, nAntenna, wl, s, xyz, d, v, nBeamReduced, scale);
  });
}
BippError bipp_eigh_gram_batched_ranked_s(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna, const float* wl,
                                          const void* s, const float* xyz, double threshold, int mode,
                                          const float* model, int margin, double residualTol, float* d, void* v,
                                          size_t* nBeamReduced, float* scale, int* kComputed, int* fallback,
                                          double* ms) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    RankOpts ro;
    ro.mode = mode;
    ro.threshold = threshold;
    ro.modelHost = model;
    ro.margin = margin;
    ro.resTol = residualTol;
    ro.kComputed = kComputed;
    ro.fallback = fallback;
    ro.ms = ms;
    eigh_gram_batched_host<float>(ctx, nBatch, nAntenna, wl, s, xyz, d, v, nBeamReduced, scale, &ro);
  });
}
BippError bipp_rank_features_s(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna, const float* wl, const void* s,
                               const float* xyz, double threshold, float* features, int* counts) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    require(features && counts, "null pointer", BIPP_INVALID_POINTER_ERROR);
    RankOpts ro;
    ro.mode = 0;
    ro.threshold = threshold;
    ro.features = features;
    std::vector<float> d(nBatch * nAntenna), sc(nBatch);
    std::vector<size_t> nr(nBatch);
    eigh_gram_batched_host<float>(ctx, nBatch, nAntenna, wl, s, xyz, d.data(), nullptr, nr.data(), sc.data(), &ro);
    for (size_t b = 0; b < nBatch; ++b) {
      int c = 0;
      for (size_t i = 0; i < nr[b]; ++i) c += (d[b * nAntenna + i] > threshold) ? 1 : 0;
      counts[b] = c;
    }
  });
}
BippError bipp_gram_matrix_s(bipp_ctx_t ctx, size_t nAntenna, size_t nBeam, const void* w, size_t ldw, const float* xyz,
                             size_t ldxyz, float wl, void* g, size_t ldg) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    gram_host<float>(ctx, nAntenna, nBeam, w, ldw, xyz, ldxyz, wl, g, ldg);
  });
}
BippError bipp_gram_matrix_d(bipp_ctx_t ctx, size_t nAntenna, size_t nBeam, const void* w, size_t ldw, const double* xyz,
                             size_t ldxyz, double wl, void* g, size_t ldg) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    gram_host<double>(ctx, nAntenna, nBeam, w, ldw, xyz, ldxyz, wl, g, ldg);
  });
}
BippError bipp_virtual_vis_s(bipp_ctx_t ctx, float scale, size_t nAntenna, size_t nBeam, const float* d, const void* v,
                             size_t ldv, void* vv) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    virtual_vis_host<float>(ctx, scale, nAntenna, nBeam, d, v, ldv, vv);
  });
}
BippError bipp_virtual_vis_d(bipp_ctx_t ctx, double scale, size_t nAntenna, size_t nBeam, const double* d, const void* v,
                             size_t ldv, void* vv) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    virtual_vis_host<double>(ctx, scale, nAntenna, nBeam, d, v, ldv, vv);
  });
}

}  // extern "C"
