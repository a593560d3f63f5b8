// C ABI of the learned rank predictor's network: forward pass, loss gradient and
// training (Adam, full batch) on the device with the hand-written kernels of
// rank_mlp.cuh. The predictor has no counterpart in the reference, which always computes
// every eigenpair (LAPACK ?hegv, src/eigensolver.cpp:188-216).
#include <cuda_runtime.h>

#include <cmath>

#include "bipp_b200.h"
#include "context.hpp"
#include "rank_mlp.cuh"

using namespace bippb200;

namespace {

struct MlpBuffers {
  DevBuf model, X, Y, H1, H2, out, grad, loss;
  MlpBuffers(bipp_ctx_s* ctx, const float* modelH, const float* XH, const float* YH, int n, int nLoss) {
    model.alloc(ctx, kMlpParams * sizeof(float));
    X.alloc(ctx, (size_t)n * kRankFeatures * sizeof(float));
    H1.alloc(ctx, (size_t)n * kMlpH * sizeof(float));
    H2.alloc(ctx, (size_t)n * kMlpH * sizeof(float));
    out.alloc(ctx, (size_t)n * sizeof(float));
    grad.alloc(ctx, kMlpParams * sizeof(float));
    loss.alloc(ctx, (size_t)std::max(1, nLoss) * sizeof(float));
    h2d(ctx, model.get(), modelH, kMlpParams * sizeof(float));
    h2d(ctx, X.get(), XH, (size_t)n * kRankFeatures * sizeof(float));
    if (YH) {
      Y.alloc(ctx, (size_t)n * sizeof(float));
      h2d(ctx, Y.get(), YH, (size_t)n * sizeof(float));
    }
  }
};

void check_model(const float* model) {
  for (int j = 0; j < kRankFeatures; ++j)
    require(std::isfinite(model[kOffSd + j]) && model[kOffSd + j] > 0.f,
            "feature standard deviations of the model must be positive");
}

}  // namespace

extern "C" {

int bipp_rank_mlp_num_params(void) { return kMlpParams; }

BippError bipp_rank_mlp_forward(bipp_ctx_t ctx, const float* model, const float* features, size_t n, float* out) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    require(model && features && out, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(n >= 1 && n <= (1u << 24), "sample count must be in [1, 2^24]");
    check_model(model);
    MlpBuffers b(ctx, model, features, nullptr, (int)n, 1);
    count_launch();
    mlp_forward_kernel<<<(int)((n + kMlpTile - 1) / kMlpTile), kMlpThreads, 0, ctx->stream>>>(
        b.model.get<float>(), b.X.get<float>(), (int)n, b.out.get<float>(), nullptr, nullptr);
    B2_CHECK_LAUNCH();
    d2h(ctx, out, b.out.get(), n * sizeof(float));
    sync(ctx);
  });
}

BippError bipp_rank_mlp_gradient(bipp_ctx_t ctx, const float* model, const float* features, const float* targets,
                                 size_t n, float* grad, float* loss) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    require(model && features && targets && grad && loss, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(n >= 1 && n <= (1u << 24), "sample count must be in [1, 2^24]");
    check_model(model);
    MlpBuffers b(ctx, model, features, targets, (int)n, 1);
    b.grad.zero();
    b.loss.zero();
    const int grid = (int)((n + kMlpTile - 1) / kMlpTile);
    count_launch();
    mlp_forward_kernel<<<grid, kMlpThreads, 0, ctx->stream>>>(b.model.get<float>(), b.X.get<float>(), (int)n,
                                                            b.out.get<float>(), b.H1.get<float>(), b.H2.get<float>());
    count_launch();
    mlp_backward_kernel<<<grid, kMlpThreads, 0, ctx->stream>>>(b.model.get<float>(), b.X.get<float>(),
                                                             b.Y.get<float>(), (int)n, b.H1.get<float>(),
                                                             b.H2.get<float>(), b.out.get<float>(), b.grad.get<float>(),
                                                             b.loss.get<float>(), nullptr);
    B2_CHECK_LAUNCH();
    d2h(ctx, grad, b.grad.get(), kMlpParams * sizeof(float));
    d2h(ctx, loss, b.loss.get(), sizeof(float));
    sync(ctx);
  });
}

BippError bipp_rank_mlp_train(bipp_ctx_t ctx, float* model, const float* features, const float* targets, size_t n,
                              int iterations, float learningRate, float* lossHistory) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    require(model && features && targets, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(n >= 1 && n <= (1u << 24), "sample count must be in [1, 2^24]");
    require(iterations >= 1 && iterations <= (1 << 24), "iterations must be in [1, 2^24]");
    require(std::isfinite(learningRate) && learningRate > 0.f, "learning rate must be positive");
    check_model(model);
    MlpBuffers b(ctx, model, features, targets, (int)n, iterations);
    DevBuf m(ctx, kMlpParams * sizeof(float)), v(ctx, kMlpParams * sizeof(float)), step(ctx, sizeof(int));
    m.zero();
    v.zero();
    step.zero();
    b.loss.zero();
    const int grid = (int)((n + kMlpTile - 1) / kMlpTile);
    const int ag = (kMlpParams + 255) / 256;
    cudaStream_t st = ctx->stream;
    // one iteration (clear the gradient, forward, backward, Adam, step counter) captured
    // once and replayed: the loop is launch bound
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    B2_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b.grad.get(), 0, kMlpParams * sizeof(float), st);
    mlp_forward_kernel<<<grid, kMlpThreads, 0, st>>>(b.model.get<float>(), b.X.get<float>(), (int)n,
                                                   b.out.get<float>(), b.H1.get<float>(), b.H2.get<float>());
    mlp_backward_kernel<<<grid, kMlpThreads, 0, st>>>(b.model.get<float>(), b.X.get<float>(), b.Y.get<float>(),
                                                    (int)n, b.H1.get<float>(), b.H2.get<float>(), b.out.get<float>(),
                                                    b.grad.get<float>(), b.loss.get<float>(), step.get<int>());
    mlp_adam_kernel<<<ag, 256, 0, st>>>(b.model.get<float>(), b.grad.get<float>(), m.get<float>(), v.get<float>(),
                                        learningRate, 0.9f, 0.999f, 1e-8f, step.get<int>());
    mlp_step_kernel<<<1, 1, 0, st>>>(step.get<int>());
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("stream capture: ") + cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    cudaError_t le = cudaSuccess;
    for (int it = 0; it < iterations && le == cudaSuccess; ++it) {
      for (int k = 0; k < 4; ++k) count_launch();
      le = cudaGraphLaunch(exec, st);
    }
    cudaGraphExecDestroy(exec);
    if (le != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("graph launch: ") + cudaGetErrorString(le));
    d2h(ctx, model, b.model.get(), kMlpParams * sizeof(float));
    if (lossHistory) d2h(ctx, lossHistory, b.loss.get(), (size_t)iterations * sizeof(float));
    sync(ctx);
  });
}

}  // extern "C"
