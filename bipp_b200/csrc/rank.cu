// C ABI of the learned rank predictor's network: forward pass, loss gradient and
// training (Adam, full batch) on the device with the hand-written kernels of
// rank_mlp.cuh. The predictor has no counterpart in the reference, which always computes
// every eigenpair (LAPACK ?hegv, src/eigensolver.cpp:188-216).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

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
                              const float* valFeatures, const float* valTargets, size_t nVal, int iterations,
                              float learningRate, float weightDecay, int evalEvery, float* lossHistory,
                              float* valHistory) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    require(model && features && targets, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(n >= 1 && n <= (1u << 24), "sample count must be in [1, 2^24]");
    require(nVal <= (1u << 24), "validation sample count above 2^24");
    require(!nVal || (valFeatures && valTargets), "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(iterations >= 1 && iterations <= (1 << 24), "iterations must be in [1, 2^24]");
    require(std::isfinite(learningRate) && learningRate > 0.f, "learning rate must be positive");
    require(std::isfinite(weightDecay) && weightDecay >= 0.f, "weight decay must be non-negative");
    require(!nVal || evalEvery >= 1, "evalEvery must be positive with a validation set");
    check_model(model);
    MlpBuffers b(ctx, model, features, targets, (int)n, iterations);
    DevBuf m(ctx, kMlpParams * sizeof(float)), v(ctx, kMlpParams * sizeof(float)), step(ctx, sizeof(int));
    DevBuf best(ctx, kMlpParams * sizeof(float)), vX, vOut;
    m.zero();
    v.zero();
    step.zero();
    b.loss.zero();
    std::vector<float> vy(nVal), vo(nVal);
    if (nVal) {
      vX.alloc(ctx, nVal * kRankFeatures * sizeof(float));
      vOut.alloc(ctx, nVal * sizeof(float));
      h2d(ctx, vX.get(), valFeatures, nVal * kRankFeatures * sizeof(float));
      std::copy(valTargets, valTargets + nVal, vy.begin());
    }
    B2_CUDA(cudaMemcpyAsync(best.get(), b.model.get(), kMlpParams * sizeof(float), cudaMemcpyDeviceToDevice,
                            ctx->stream));
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
                                        learningRate, 0.9f, 0.999f, 1e-8f, weightDecay, step.get<int>());
    mlp_step_kernel<<<1, 1, 0, st>>>(step.get<int>());
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (ce != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("stream capture: ") + cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(ie));
    // validation loss of the current model (host), every evalEvery iterations; the model
    // with the lowest one is kept
    auto val_loss = [&]() {
      count_launch();
      mlp_forward_kernel<<<(int)((nVal + kMlpTile - 1) / kMlpTile), kMlpThreads, 0, st>>>(
          b.model.get<float>(), vX.get<float>(), (int)nVal, vOut.get<float>(), nullptr, nullptr);
      B2_CHECK_LAUNCH();
      d2h(ctx, vo.data(), vOut.get(), nVal * sizeof(float));
      sync(ctx);
      double l = 0;
      for (size_t i = 0; i < nVal; ++i) l += ((double)vo[i] - vy[i]) * ((double)vo[i] - vy[i]);
      return l / (double)nVal;
    };
    double bestVal = nVal ? val_loss() : 0.0;
    int evals = 0;
    cudaError_t le = cudaSuccess;
    try {
      for (int it = 0; it < iterations && le == cudaSuccess; ++it) {
        for (int k = 0; k < 4; ++k) count_launch();
        le = cudaGraphLaunch(exec, st);
        if (le == cudaSuccess && nVal && ((it + 1) % evalEvery == 0 || it + 1 == iterations)) {
          const double l = val_loss();
          if (valHistory) valHistory[evals] = (float)l;
          ++evals;
          if (l < bestVal) {
            bestVal = l;
            B2_CUDA(cudaMemcpyAsync(best.get(), b.model.get(), kMlpParams * sizeof(float), cudaMemcpyDeviceToDevice,
                                    st));
          }
        }
      }
    } catch (...) {
      cudaGraphExecDestroy(exec);
      throw;
    }
    cudaGraphExecDestroy(exec);
    if (le != cudaSuccess) throw Error(BIPP_GPU_ERROR, std::string("graph launch: ") + cudaGetErrorString(le));
    d2h(ctx, model, nVal ? best.get() : b.model.get(), kMlpParams * sizeof(float));
    if (lossHistory) d2h(ctx, lossHistory, b.loss.get(), (size_t)iterations * sizeof(float));
    sync(ctx);
  });
}

}  // extern "C"
