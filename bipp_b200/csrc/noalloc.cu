// eigh_gram for one time step that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc/cudaFree: an imager embedded in a
// host framework whose caching allocator owns all of the device memory (a foreign
// cudaMalloc can fail or fragment that pool), or a real-time correlator/beamformer loop
// that must not block, since cudaFree waits for the whole device to go idle. For them
// this entry point runs the same eigensolver kernels as bipp_eigh_gram_s on
// caller-provided device inputs and outputs, with every intermediate matrix in one
// file-scope __device__ array of fixed size (see kNoAllocScratchBytes below).
#include <cuda_runtime.h>

#include <cfloat>
#include <climits>

#include "bipp_b200.h"
#include "context.hpp"
#include "eig_kernels.cuh"

namespace bippb200 {
namespace {

constexpr int kN = BIPP_NOALLOC_MAX_ANTENNA;
constexpr size_t al256(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t kN2 = (size_t)kN * kN;
// eigensolver workspace of one matrix of size kN (float path), as carve() lays it out
constexpr size_t kWorkBytes = al256(kN2 * sizeof(float2)) * 3 + al256(kN2 * sizeof(double2)) * 2 +
                              al256(kN2 * sizeof(float)) + al256(kN * sizeof(double)) * 2 + al256(kN * sizeof(float2));
// per-step arrays: idx, nred, nvis, status, lam, wl
constexpr size_t kOffIdx = kWorkBytes;
constexpr size_t kOffNred = kOffIdx + al256(kN * sizeof(int));
constexpr size_t kOffNvis = kOffNred + 256;
constexpr size_t kOffStatus = kOffNvis + 256;
constexpr size_t kOffLam = kOffStatus + 256;
constexpr size_t kOffWl = kOffLam + al256(kN * sizeof(double));
constexpr size_t kNoAllocScratchBytes = kOffWl + 256;

// Shared by every call on a device and kept until the process exits; holds the last
// call's intermediates (calls that overlap on the GPU race on it).
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of the scratch array in the current device's context. The host-side
// symbol is only a stand-in, not a device address; the lookup allocates nothing and is
// repeated on every call, so a context that was re-created (cudaDeviceReset) never leaves
// a stale address behind.
void* scratch_address() {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  return p;
}

// makes `device` current for the call and gives the caller's current device back on
// every exit path (the caller may be a framework with its own notion of the current GPU)
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int device) {
    B2_CUDA(cudaGetDevice(&prev));
    if (prev != device) B2_CUDA(cudaSetDevice(device));
  }
  ~DeviceScope() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

struct Work {
  float2 *A, *Linv, *T1;
  double2 *G, *W64;
  float* Z;
  double *d, *e;
  float2* tau;
};

// workspace of one N x N problem (N <= kN) inside the scratch array
Work carve(char* base, int N) {
  const size_t n2 = (size_t)N * N;
  Work w;
  char* p = base;
  w.A = reinterpret_cast<float2*>(p); p += al256(n2 * sizeof(float2));
  w.Linv = reinterpret_cast<float2*>(p); p += al256(n2 * sizeof(float2));
  w.T1 = reinterpret_cast<float2*>(p); p += al256(n2 * sizeof(float2));
  w.G = reinterpret_cast<double2*>(p); p += al256(n2 * sizeof(double2));
  w.W64 = reinterpret_cast<double2*>(p); p += al256(n2 * sizeof(double2));
  w.Z = reinterpret_cast<float*>(p); p += al256(n2 * sizeof(float));
  w.d = reinterpret_cast<double*>(p); p += al256(N * sizeof(double));
  w.e = reinterpret_cast<double*>(p); p += al256(N * sizeof(double));
  w.tau = reinterpret_cast<float2*>(p);
  return w;
}

// outputs: d (float, zero padded), v = eigenvectors scattered to the kept antenna rows,
// nReduced, scale = 1/nVis, info (1 when the Cholesky factorisation of G failed, a kept
// entry of S is not finite, or every row and column is flagged)
__global__ void noalloc_outputs_kernel(int n, const int* __restrict__ nredP, const long long* __restrict__ nvisP,
                                       const int* __restrict__ status, const double* __restrict__ lam,
                                       const float2* __restrict__ X, int Nmax, const int* __restrict__ idx,
                                       float* __restrict__ d, float2* __restrict__ v, long long ldv,
                                       int* __restrict__ nReduced, float* __restrict__ scale, int* __restrict__ info) {
  const int nred = *nredP;
  const long long tid = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long c = tid; c < n; c += stride) d[c] = (c < nred) ? (float)lam[c] : 0.0f;
  for (long long e = tid; e < (long long)n * n; e += stride) {
    const int a = (int)(e % n), c = (int)(e / n);
    float2 val = make_float2(0.f, 0.f);
    if (c < nred) {
      int lo = 0, hi = nred;
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (idx[mid] < a) lo = mid + 1; else hi = mid;
      }
      if (lo < nred && idx[lo] == a) val = X[lo + (long long)c * Nmax];
    }
    v[a + (long long)c * ldv] = val;
  }
  if (tid == 0) {
    *nReduced = nred;
    const long long nv = *nvisP;
    *scale = nv ? 1.0f / (float)nv : 0.0f;
    *info = ((*status & (kStatusCholeskyNotPD | kStatusNonFinite)) || nred == 0) ? 1 : 0;
  }
}

__global__ void noalloc_wl_kernel(double* __restrict__ out, double wl) { *out = wl; }

}  // namespace
}  // namespace bippb200

using namespace bippb200;

extern "C" BippError bipp_eigh_gram_noalloc_s(int device, void* stream, float wl, size_t nAntenna, const void* s,
                                              size_t lds, const double* xyz, size_t ldxyz, float* d, void* v,
                                              size_t ldv, int* nBeamReduced, float* scale, int* info) {
  return guard([&] {
    require(s && xyz && d && v && nBeamReduced && scale && info, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(nAntenna >= 1, "empty problem");
    require(nAntenna <= (size_t)kN,
            "bipp_eigh_gram_noalloc_s: nAntenna exceeds BIPP_NOALLOC_MAX_ANTENNA (use bipp_eigh_gram_s)");
    require(lds >= nAntenna && ldxyz >= nAntenna && ldv >= nAntenna, "invalid leading dimension");
    require(lds <= (size_t)INT_MAX && ldxyz <= (size_t)INT_MAX, "leading dimension above INT_MAX");
    int nDev = 0;
    B2_CUDA(cudaGetDeviceCount(&nDev));
    require(device >= 0 && device < nDev, "invalid device id");
    DeviceScope scope(device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* base = static_cast<char*>(scratch_address());
    const int N = (int)nAntenna;
    const Work w = carve(base, N);
    int* idx = reinterpret_cast<int*>(base + kOffIdx);
    int* nred = reinterpret_cast<int*>(base + kOffNred);
    long long* nvis = reinterpret_cast<long long*>(base + kOffNvis);
    int* status = reinterpret_cast<int*>(base + kOffStatus);
    double* lam = reinterpret_cast<double*>(base + kOffLam);
    double* wlD = reinterpret_cast<double*>(base + kOffWl);
    // the array keeps the previous call's contents: clear the status word
    B2_CUDA(cudaMemsetAsync(status, 0, sizeof(int), st));
    noalloc_wl_kernel<<<1, 1, 0, st>>>(wlD, (double)wl);
    B2_CHECK_LAUNCH();
    // the eigensolver kernel sequence of bipp_eigh_gram_s (W = I), on the scratch array
    const long long n2 = (long long)N * N;
    const int tiles = (N + kGemmBM - 1) / kGemmBM;
    prep_kernel<float><<<1, kPrepThreads, 2 * (size_t)N * sizeof(int), st>>>(
        N, static_cast<const float2*>(s), 0, (int)lds, xyz, 0, (int)ldxyz, wlD, 0, FLT_EPSILON, 1, N, idx, nred, nvis,
        w.A, w.G, status, 1, 1, 0);
    smem_optin(cholesky_kernel<double2>, kCholSmem);
    cholesky_kernel<double2><<<1, kCholThreads, kCholSmem, st>>>(w.G, nred, N, status);
    smem_optin(trinv_kernel<double2, float2>, kTrinvSmem);
    trinv_kernel<double2, float2><<<1, 256, kTrinvSmem, st>>>(w.G, w.W64, w.Linv, nred, N);
    GemmArgs<float2> g1{};
    g1.A = w.Linv; g1.strideA = n2; g1.lda = N; g1.opA = 0;
    g1.B = w.A; g1.strideB = n2; g1.ldb = N; g1.opB = 0;
    g1.Cm = w.T1; g1.strideC = n2; g1.ldc = N;
    g1.n = nred; g1.triA = 1; g1.outMode = 0; g1.levels = 1;
    gemm_kernel<float2, float><<<dim3(tiles, tiles, 1), kGemmThreads, 0, st>>>(g1);
    GemmArgs<float2> g2{};
    g2.A = w.T1; g2.strideA = n2; g2.lda = N; g2.opA = 0;
    g2.B = w.Linv; g2.strideB = n2; g2.ldb = N; g2.opB = 1;
    g2.Cm = w.A; g2.strideC = n2; g2.ldc = N;
    g2.n = nred; g2.triB = 1; g2.outMode = 1; g2.levels = 1;
    gemm_kernel<float2, float><<<dim3(tiles, tiles, 1), kGemmThreads, 0, st>>>(g2);
    B2_CHECK_LAUNCH();
    {
      const size_t smem = hetrd_smem_bytes(N, sizeof(float2));
      smem_optin(hetrd_kernel<float2, float>, smem);
      hetrd_kernel<float2, float><<<1, trd_threads(N), smem, st>>>(w.A, nred, N, w.d, w.e, w.tau);
    }
    {
      const size_t smem = 4 * (size_t)N * sizeof(double);
      smem_optin(tridiag_kernel<float>, smem);
      tridiag_kernel<float><<<1, kTriThreads, smem, st>>>(w.d, w.e, nred, N, lam, w.Z,
                                                           reinterpret_cast<double*>(w.W64), status);
    }
    {
      const size_t smem = ((size_t)N * 16 + N + kBtThreads) * sizeof(float2);
      smem_optin(backtransform_kernel<float2, float, 16>, smem);
      backtransform_kernel<float2, float, 16><<<dim3((N + 15) / 16, 1), kBtThreads, smem, st>>>(w.A, w.tau, w.Z, nred,
                                                                                               N, w.T1, nullptr);
    }
    GemmArgs<float2> g3{};
    g3.A = w.Linv; g3.strideA = n2; g3.lda = N; g3.opA = 1;
    g3.B = w.T1; g3.strideB = n2; g3.ldb = N; g3.opB = 0;
    g3.Cm = reinterpret_cast<float2*>(w.G); g3.strideC = n2; g3.ldc = N;
    g3.n = nred; g3.triA = 2; g3.outMode = 0; g3.levels = 1;
    gemm_kernel<float2, float><<<dim3(tiles, tiles, 1), kGemmThreads, 0, st>>>(g3);
    B2_CHECK_LAUNCH();
    noalloc_outputs_kernel<<<64, 256, 0, st>>>(N, nred, nvis, status, lam, reinterpret_cast<const float2*>(w.G), N, idx,
                                               d, static_cast<float2*>(v), (long long)ldv, nBeamReduced, scale, info);
    B2_CHECK_LAUNCH();
  });
}
