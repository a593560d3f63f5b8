// Shared device helpers for the Bluebild sm_100a kernels: complex arithmetic on
// float2/double2, block reductions, error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <stdexcept>
#include <string>

#include "bipp_b200.h"

namespace bippb200 {

// ---- error handling --------------------------------------------------------------

struct Error : std::runtime_error {
  BippError code;
  Error(BippError c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

#define B2_CUDA(call)                                                                   \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::bippb200::Error(BIPP_GPU_ERROR, std::string(#call) + ": " +               \
                                                  cudaGetErrorString(e_));              \
  } while (0)

#define B2_CHECK_LAUNCH() B2_CUDA(cudaGetLastError())

// Count of kernel launches issued by this library (read by bipp_kernel_launch_count);
// every launch site calls count_launch() right before its <<<>>>.
void count_launch();

inline void require(bool ok, const char* msg, BippError code = BIPP_INVALID_PARAMETER_ERROR) {
  if (!ok) throw Error(code, msg);
}

// Per-matrix status bits written by kernels and read back by the host.
enum StatusBits : int {
  kStatusCholeskyNotPD = 1,   // non-positive pivot in the FP64 Cholesky of G
  kStatusNonFinite = 2,       // NaN/Inf in an entry of S that enters the reduced matrix
  kStatusClusterFix = 4,      // eigenvector cluster re-orthogonalised (informational)
  kStatusTensorTimeout = 8,   // a tensor-core MMA completion wait ran out (GPU error)
  kStatusRankFallback = 16,   // predicted partial solve fell back to the full solve (informational)
  kStatusResidual = 32,       // an eigenpair residual above the requested tolerance
};

// ---- complex helpers --------------------------------------------------------------

template <typename T> struct Cplx;
template <> struct Cplx<float> { using type = float2; };
template <> struct Cplx<double> { using type = double2; };

__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return mk(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 operator+(double2 a, double2 b) { return mk(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 operator-(double2 a, double2 b) { return mk(a.x - b.x, a.y - b.y); }

template <typename C> __host__ __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename C> __host__ __device__ __forceinline__ C cmulc(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
template <typename C> __host__ __device__ __forceinline__ C cconjmul(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
template <typename C> __host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <typename C, typename R> __host__ __device__ __forceinline__ C cscale(C a, R s) {
  return mk(a.x * s, a.y * s);
}
// acc += a * b
template <typename C> __host__ __device__ __forceinline__ void cfma(C& acc, C a, C b) {
  acc.x = fma(a.x, b.x, fma(-a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(a.y, b.x, acc.y));
}
// acc += conj(a) * b
template <typename C> __host__ __device__ __forceinline__ void cfma_cj(C& acc, C a, C b) {
  acc.x = fma(a.x, b.x, fma(a.y, b.y, acc.x));
  acc.y = fma(a.x, b.y, fma(-a.y, b.x, acc.y));
}
template <typename C> __host__ __device__ __forceinline__ auto cabs2(C a) { return a.x * a.x + a.y * a.y; }
// |s|^2 of the flag test as the reference's std::norm: both products and the sum rounded
// separately (no fused multiply-add), so that keep/drop matches it bit for bit
__device__ __forceinline__ float flag_norm(float2 a) { return __fadd_rn(__fmul_rn(a.x, a.x), __fmul_rn(a.y, a.y)); }
__device__ __forceinline__ double flag_norm(double2 a) { return __dadd_rn(__dmul_rn(a.x, a.x), __dmul_rn(a.y, a.y)); }

__device__ __forceinline__ float2 to_f(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ double2 to_d(float2 a) { return make_double2(a.x, a.y); }

// ---- reductions ----------------------------------------------------------------------

template <typename T> __device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T> __device__ __forceinline__ T warp_max(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
template <typename T> __device__ __forceinline__ T warp_min(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Block-wide sum; `scratch` needs blockDim.x/32 elements. Result broadcast to all threads.
template <typename T> __device__ __forceinline__ T block_sum(T v, T* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  T r = (lane < nw) ? scratch[lane] : T(0);
  r = warp_sum(r);
  return r;
}
template <typename T> __device__ __forceinline__ T block_max(T v, T* scratch, T init) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_max(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  T r = (lane < nw) ? scratch[lane] : init;
  return warp_max(r);
}
template <typename T> __device__ __forceinline__ T block_min(T v, T* scratch, T init) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_min(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  T r = (lane < nw) ? scratch[lane] : init;
  return warp_min(r);
}

inline int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace bippb200
