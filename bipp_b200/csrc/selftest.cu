// Self-test of the bounded waits of the tensor-core kernels (no counterpart in the
// reference). Every wait of this library on an MMA completion barrier gives up after a
// spin limit, records the timeout in a status word and lets the kernel release its
// resources, so that a stuck tensor-core operation reaches the caller as BIPP_GPU_ERROR
// instead of a hang. This entry point runs that wait on a barrier that nothing ever
// completes, with the caller's spin limit, so that the path can be exercised without
// any fault.
#include <cuda_runtime.h>

#include "bipp_b200.h"
#include "context.hpp"
#include "tc_common.cuh"

namespace bippb200 {
namespace {

__global__ void wait_timeout_kernel(int spins, int* __restrict__ status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) mbar_init(smem_u32(&bar), 1);
  __syncthreads();
  if (threadIdx.x == 0) status[0] = mbar_wait(smem_u32(&bar), 0u, spins) ? 0 : (int)kStatusTensorTimeout;
}

}  // namespace
}  // namespace bippb200

using namespace bippb200;

extern "C" BippError bipp_selftest_wait_timeout(bipp_ctx_t ctx, int spins, int* timedOut) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    require(timedOut != nullptr, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(spins >= 1 && spins <= (1 << 20), "spin limit must be in [1, 2^20]");
    DevBuf st(ctx, sizeof(int));
    st.zero();
    count_launch();
    wait_timeout_kernel<<<1, 32, 0, ctx->stream>>>(spins, st.get<int>());
    B2_CHECK_LAUNCH();
    int h = 0;
    d2h(ctx, &h, st.get(), sizeof(int));
    sync(ctx);
    *timedOut = (h & kStatusTensorTimeout) ? 1 : 0;
    if (*timedOut) throw Error(BIPP_GPU_ERROR, "tensor-core barrier wait timed out (self-test)");
  });
}
