// Batched eigensolver workspace and launch descriptor shared by the eigensolver
// entry points and the synthesis pipeline.
#pragma once

#include "common.cuh"
#include "context.hpp"

namespace bippb200 {

template <typename T>
struct EigWork {
  int capBatch = 0, Nmax = 0;
  DevBuf A, G, W64, Linv, T1, Z, d, e, tau, krange, order;
  void reserve(bipp_ctx_s* ctx, int nBatch, int Nmax);
  // compacted eigenvectors (column c = eigenvector of eigenvalue c), ld Nmax
  typename Cplx<T>::type* X(bool gram);
};

template <typename T>
struct EigLaunch {
  int nBatch = 0;      // matrices in this launch
  int nBeam = 0;       // rows/cols of S
  int nAnt = 0;        // antennas (general W only)
  int Nmax = 0;        // padded size (>= nBeam)
  const typename Cplx<T>::type* S = nullptr;  // first matrix of this launch
  long long sStride = 0;
  int lds = 0;
  const double* xyz = nullptr;  // positions of all matrices ([batch][3][ldxyz] via xyzStride)
  long long xyzStride = 0;
  int ldxyz = 0;
  const double* wl = nullptr;   // [batch]
  double hostWl = 0;
  int mode = 0;                 // 0 eigh_gram flag test, 1 eigh flag test
  T eps = 0;
  bool gram = true;
  bool identityW = true;
  const typename Cplx<T>::type* W = nullptr;  // general W (single matrix)
  int ldw = 0;
  int hostNred = 0;             // nred of the single matrix (general W)
  // per-matrix outputs indexed by batchOffset + b
  int* idx = nullptr;           // [batch][Nmax]
  int* nred = nullptr;          // [batch]
  long long* nvis = nullptr;    // [batch]
  int* status = nullptr;        // [batch]
  double* lam = nullptr;        // [batch][Nmax]
  int doFlag = 1;
  int batchOffset = 0;
  // eigenvectors are needed only for eigenvalues in [vecLo, vecHi] (the synthesis uses
  // those inside its energy levels); the others are returned as zero columns
  double vecLo = -1.0 / 0.0, vecHi = 1.0 / 0.0;
  // 0: eigenvalues outside [vecLo, vecHi] are not computed either (returned as zero)
  int allValues = 1;
  // optional per-kernel device time accumulation (ms): prep, cholesky, trinv, reduction
  // GEMMs, hetrd, tridiagonal eigenpairs, back-transform, Linv^H Y GEMM
  double* kernelMs = nullptr;
  // rank predictor (optional): the features ([batch][64], device) of the whitened matrix,
  // formed after the reduction with featThreshold as the energy threshold; with mlpModel
  // (device) the MLP predicts the count of eigenvalues above vecLo (mlpOut [batch]
  // fractions, predK [batch] counts) and the tridiagonal stage computes the largest
  // predK + predMargin eigenpairs, falling back to all of them when the smallest computed
  // value is still above vecLo or (resTol >= 0) a residual exceeds resTol |T|
  float* features = nullptr;
  double featThreshold = 0.0;
  const float* mlpModel = nullptr;
  float* mlpOut = nullptr;
  int* predK = nullptr;
  int predMargin = 16;
  double resTol = -1.0;
};

constexpr int kEigTimers = 8;

// options of the ranked batched eigh_gram (single precision): mode 0 computes every
// eigenpair, 1 those above `threshold` (exact index range by Sturm counts), 2 the largest
// k + margin with k predicted by the MLP `modelHost` (host, kMlpParams floats), falling
// back to every eigenpair when needed; optional outputs per step: the features
// ([nBatch][64]), the number of eigenvectors computed, the fallback flag, and the
// device time of the eigensolver launches
struct RankOpts {
  int mode = 0;
  double threshold = 0.0;
  const float* modelHost = nullptr;
  int margin = 16;
  double resTol = -1.0;
  float* features = nullptr;
  int* kComputed = nullptr;
  int* fallback = nullptr;
  double* ms = nullptr;
};

template <typename T>
void eig_launch(bipp_ctx_s* ctx, const EigLaunch<T>& L, EigWork<T>& w);

}  // namespace bippb200
