// Internal context: one CUDA device, one non-blocking stream, stream-ordered device
// allocations (cudaMallocAsync pool) and cached kernel attributes. Mirrors the role of
// the reference's ContextInternal + gpu::Queue (src/context_internal.hpp:24-54,
// src/gpu/util/queue.hpp:20-58): every API call runs on the context's stream and is
// synchronous on return.
#pragma once

#include <atomic>

#include <cuda_runtime.h>

#include <cstring>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "bipp_b200.h"
#include "common.cuh"

struct bipp_ctx_s {
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaDeviceProp prop{};
  int smCount = 0;
  size_t maxSmemOptin = 0;
  // references: the caller's (dropped by bipp_ctx_destroy) and one per live pipeline or
  // NUFFT collector created on it, so that the context outlives them whatever the order
  // of the destroy calls
  std::atomic<int> refs{1};
};

namespace bippb200 {

void set_last_error(const std::string& msg);

// a pipeline or collector keeps its context alive
inline void ctx_retain(bipp_ctx_s* c) { c->refs.fetch_add(1); }
// drop a reference; the last one synchronises and frees the context
void ctx_release(bipp_ctx_s* c);

// RAII device buffer on the context's stream-ordered pool.
class DevBuf {
public:
  DevBuf() = default;
  DevBuf(bipp_ctx_s* ctx, size_t bytes) { alloc(ctx, bytes); }
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ctx_ = o.ctx_;
      ptr_ = o.ptr_;
      bytes_ = o.bytes_;
      o.ptr_ = nullptr;
      o.bytes_ = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(bipp_ctx_s* ctx, size_t bytes) {
    release();
    ctx_ = ctx;
    bytes_ = bytes;
    if (bytes) B2_CUDA(cudaMallocAsync(&ptr_, bytes, ctx->stream));
  }
  // grow-only reallocation (contents not preserved)
  void ensure(bipp_ctx_s* ctx, size_t bytes) {
    if (bytes > bytes_ || !ptr_) alloc(ctx, bytes);
  }
  void release() {
    if (ptr_ && ctx_) cudaFreeAsync(ptr_, ctx_->stream);
    ptr_ = nullptr;
    bytes_ = 0;
  }
  template <typename T = void> T* get() const { return reinterpret_cast<T*>(ptr_); }
  size_t bytes() const { return bytes_; }
  void zero() {
    if (ptr_) B2_CUDA(cudaMemsetAsync(ptr_, 0, bytes_, ctx_->stream));
  }

private:
  bipp_ctx_s* ctx_ = nullptr;
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
};

// Host <-> device helpers on the context stream.
inline void h2d(bipp_ctx_s* c, void* dst, const void* src, size_t bytes) {
  if (bytes) B2_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
}
inline void d2h(bipp_ctx_s* c, void* dst, const void* src, size_t bytes) {
  if (bytes) B2_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
}
inline void sync(bipp_ctx_s* c) { B2_CUDA(cudaStreamSynchronize(c->stream)); }

// Allow a kernel to use large dynamic shared memory (dynamic + static above 48 KB needs
// the opt-in, so it is requested for anything above 32 KB of dynamic memory).
template <typename K>
inline void smem_optin(K kernel, size_t bytes) {
  if (bytes > 32 * 1024) B2_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
}

// Run an API body, translating exceptions into BippError codes.
BippError guard(const std::function<void()>& body);

}  // namespace bippb200
