/*
 * bipp_b200.h - C ABI of the B200-native Bluebild imaging path.
 *
 * Every entry point takes plain pointers and sizes and returns a BippError. Array
 * layouts are those of the reference API: column-major with leading dimensions,
 * complex values as interleaved (re, im) pairs (std::complex layout), uvw and lmn as
 * (n x 3) column-major, i.e. three separate coordinate arrays. Unless stated
 * otherwise pointers are host pointers and calls are synchronous on return.
 * After a failure, bipp_last_error() returns a message for the calling thread.
 *
 * Reference interfaces replaced (paths relative to the reference project):
 *   Context                       include/bipp/context.hpp:17-76, src/context_internal.cpp:27-73
 *   eigh / eigh_gram              include/bipp/bipp.hpp:47-75, src/eigensolver.cpp:40-225
 *   host::gram_matrix             src/host/gram_matrix.hpp:15-17
 *   host::virtual_vis             src/host/virtual_vis.hpp:15-17
 *   nuft_sum (host and GPU)       src/host/kernels/nuft_sum.hpp, src/gpu/kernels/nuft_sum.hpp
 *   NUFFTInterface add/get_image  src/nufft_interface.hpp:13-21, src/gpu/nufft.hpp:28-235
 *   DomainPartition::grid         src/host/domain_partition.hpp:35-101
 *   image_synthesis               include/bipp/image_synthesis.hpp:160-163, src/image_synthesis.cpp:28-182
 */
#pragma once

#include <stddef.h>

#include "bipp/enums.h"
#include "bipp/errors.h"

#ifdef __cplusplus
extern "C" {
#endif

#define BIPP_B200_EXPORT __attribute__((visibility("default")))

typedef struct bipp_ctx_s* bipp_ctx_t;
typedef struct bipp_nufft_s* bipp_nufft_t;
typedef struct bipp_pipeline_s* bipp_pipeline_t;

/* Message of the last failed call on this thread (empty if none). */
BIPP_B200_EXPORT const char* bipp_last_error(void);

/* Number of this library's own CUDA kernels launched by this process so far (all
 * threads and devices; cuFFT's kernels are not counted). No reference counterpart:
 * an instrumentation hook for benchmarks (launches between two reads = difference). */
BIPP_B200_EXPORT unsigned long long bipp_kernel_launch_count(void);

/* ---- context ------------------------------------------------------------------- */

/* Create a context on the current CUDA device (replaces Context(BippProcessingUnit),
 * include/bipp/context.hpp:25). BIPP_PU_AUTO and BIPP_PU_GPU select the GPU;
 * BIPP_PU_CPU is rejected with BIPP_INVALID_PARAMETER_ERROR: this library has no CPU
 * path. Fails with BIPP_GPU_SUPPORT_ERROR when no CUDA device is present. */
BIPP_B200_EXPORT BippError bipp_ctx_create(BippProcessingUnit pu, bipp_ctx_t* ctx);
/* As bipp_ctx_create on an explicit device (the reference picks rank % deviceCount,
 * src/context_internal.cpp:59-66). */
BIPP_B200_EXPORT BippError bipp_ctx_create_on_device(BippProcessingUnit pu, int device, bipp_ctx_t* ctx);
/* Drops the caller's reference: pipelines and NUFFT collectors created on the context
 * keep it alive until they are destroyed, so the destroy calls may come in any order. */
BIPP_B200_EXPORT BippError bipp_ctx_destroy(bipp_ctx_t ctx);
/* Processing unit actually used (always BIPP_PU_GPU). Context::processing_unit(),
 * include/bipp/context.hpp:60. */
BIPP_B200_EXPORT BippError bipp_ctx_processing_unit(bipp_ctx_t ctx, BippProcessingUnit* pu);
/* CUDA stream used by the context (as void*, a cudaStream_t). */
BIPP_B200_EXPORT BippError bipp_ctx_stream(bipp_ctx_t ctx, void** stream);

/* ---- eigensolvers ----------------------------------------------------------------- */

/* Generalized eigenproblem S x = d G x with G the beamformed Gram matrix of the
 * antenna positions; replaces bipp::eigh_gram<float/double> (include/bipp/bipp.hpp:70-75,
 * src/eigensolver.cpp:129-225). s: nBeam x nBeam (lower triangle used), w: nAntenna x
 * nBeam, xyz: nAntenna x 3. Outputs d[nBeam] ascending, zero padded; v nAntenna x nBeam
 * zero padded; *nBeamReduced and *scale = 1/nVis as the reference's returned pair.
 * Errors as the reference's LAPACK ?hegv (src/host/lapack_api.hpp:112-158, info != 0 ->
 * EigensolverError): BIPP_EIGENSOLVER_ERROR when G is not positive definite or when a
 * NaN/Inf entry of S's lower triangle lies in a kept row and column. A NaN/Inf entry fails
 * the flag test like a zero, so an antenna whose entries are all NaN is dropped, and
 * entries above the diagonal are never read. A step whose rows and columns are all
 * flagged fails with BIPP_EIGENSOLVER_ERROR after zeroing d and v (the reference's LAPACK
 * call rejects the empty problem's leading dimension 0). nBeam is at most 4096 for the _s entry
 * points and, for _d, at most the FP64 limit set by the device's shared memory per block
 * (2854 on B200); larger problems fail with BIPP_INVALID_PARAMETER_ERROR. */
BIPP_B200_EXPORT BippError bipp_eigh_gram_s(bipp_ctx_t ctx, float wl, size_t nAntenna, size_t nBeam,
                                            const void* s, size_t lds, const void* w, size_t ldw,
                                            const float* xyz, size_t ldxyz, float* d, void* v, size_t ldv,
                                            size_t* nBeamReduced, float* scale);
BIPP_B200_EXPORT BippError bipp_eigh_gram_d(bipp_ctx_t ctx, double wl, size_t nAntenna, size_t nBeam,
                                            const void* s, size_t lds, const void* w, size_t ldw,
                                            const double* xyz, size_t ldxyz, double* d, void* v, size_t ldv,
                                            size_t* nBeamReduced, double* scale);

/* Standard Hermitian eigenproblem of S; replaces bipp::eigh<float/double>
 * (include/bipp/bipp.hpp:47-51, src/eigensolver.cpp:40-127). Non-finite entries as for
 * bipp_eigh_gram_s (the reference's ?heev, src/host/lapack_api.hpp:70-110). */
BIPP_B200_EXPORT BippError bipp_eigh_s(bipp_ctx_t ctx, float wl, size_t nAntenna, size_t nBeam, const void* s,
                                       size_t lds, const void* w, size_t ldw, float* d, void* v, size_t ldv,
                                       size_t* nBeamReduced, float* scale);
BIPP_B200_EXPORT BippError bipp_eigh_d(bipp_ctx_t ctx, double wl, size_t nAntenna, size_t nBeam, const void* s,
                                       size_t lds, const void* w, size_t ldw, double* d, void* v, size_t ldv,
                                       size_t* nBeamReduced, double* scale);

/* Batched eigh_gram with W = I (nBeam = nAntenna) over nBatch independent time steps,
 * one launch sequence for the whole batch. The per-step loop of the reference's
 * dataset creation (python/bipp/apps/create_dataset.py:78-103) calls eigh_gram once per
 * step; this is its batched form. s: [nBatch][nAntenna x nAntenna] (lds = nAntenna),
 * xyz: [nBatch][nAntenna x 3], wl: [nBatch]; d: [nBatch][nAntenna], v: [nBatch][nAntenna x
 * nAntenna]; nBeamReduced, scale: [nBatch]. Fails as bipp_eigh_gram_s when any step
 * fails. */
BIPP_B200_EXPORT BippError bipp_eigh_gram_batched_s(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna,
                                                    const float* wl, const void* s, const float* xyz, float* d,
                                                    void* v, size_t* nBeamReduced, float* scale);
/* FP64 form of bipp_eigh_gram_batched_s (the reference's eigh_gram<double>, zhegv, per
 * step): complex double s and v, double wl, xyz, d and scale; nAntenna at most the FP64
 * limit of bipp_eigh_gram_d. */
BIPP_B200_EXPORT BippError bipp_eigh_gram_batched_d(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna,
                                                    const double* wl, const void* s, const double* xyz, double* d,
                                                    void* v, size_t* nBeamReduced, double* scale);

/* ---- learned rank predictor --------------------------------------------------------- */
/* No counterpart in the reference, which computes every eigenpair (LAPACK ?hegv,
 * src/eigensolver.cpp:188-216) and keeps those inside the energy levels afterwards.
 *
 * Ranked form of bipp_eigh_gram_batched_s (same inputs and outputs): mode 0 computes every
 * eigenpair (the reference's full solve); mode 1 the eigenpairs above `threshold`, their
 * index range found exactly by Sturm counts of the tridiagonal matrix; mode 2 the largest
 * k + margin, with k, the count above the threshold, predicted per step by the MLP `model`
 * (host, bipp_rank_mlp_num_params() floats) from the features of the whitened matrix. Mode
 * 2 falls back to every eigenpair of a step when its smallest computed eigenvalue is still
 * above the threshold (eigenvalues above it may be missing) or, with residualTol >= 0, when
 * a computed pair has |T z - d z|_inf > residualTol |T| |z|_inf (T the tridiagonal matrix).
 * Eigenvalues and eigenvectors not computed are returned as zero. Optional outputs per
 * step: kComputed (eigenvectors computed), fallback (1 if the step fell back); ms: device
 * time of the eigensolver kernels. */
BIPP_B200_EXPORT BippError bipp_eigh_gram_batched_ranked_s(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna,
                                                           const float* wl, const void* s, const float* xyz,
                                                           double threshold, int mode, const float* model, int margin,
                                                           double residualTol, float* d, void* v,
                                                           size_t* nBeamReduced, float* scale, int* kComputed,
                                                           int* fallback, double* ms);
/* Training data of the predictor from the method itself: the full solve of each step (as
 * bipp_eigh_gram_batched_s) with the 64 features of its whitened matrix L^-1 S L^-H
 * (features [nBatch][64]) and the count of eigenvalues above `threshold` (counts [nBatch]). */
BIPP_B200_EXPORT BippError bipp_rank_features_s(bipp_ctx_t ctx, size_t nBatch, size_t nAntenna, const float* wl,
                                                const void* s, const float* xyz, double threshold, float* features,
                                                int* counts);
/* Floats of an MLP model (64 -> 128 -> 128 -> 1, ReLU): feature mean [64], standard
 * deviation [64], W1 [64][128], b1 [128], W2 [128][128], b2 [128], W3 [128], b3. */
BIPP_B200_EXPORT int bipp_rank_mlp_num_params(void);
/* out[i] = MLP((features[i] - mean) / sd), features [n][64] (host pointers). */
BIPP_B200_EXPORT BippError bipp_rank_mlp_forward(bipp_ctx_t ctx, const float* model, const float* features, size_t n,
                                                 float* out);
/* Gradient of the loss (1/n) sum_i (out_i - targets_i)^2 with respect to every model
 * float (zero for the fixed mean and sd), and the loss. */
BIPP_B200_EXPORT BippError bipp_rank_mlp_gradient(bipp_ctx_t ctx, const float* model, const float* features,
                                                  const float* targets, size_t n, float* grad, float* loss);
/* Train the model in place on the device: `iterations` full-batch Adam steps (beta 0.9,
 * 0.999, eps 1e-8) on the loss above plus the L2 penalty (weightDecay / 2) |W|^2 of the
 * weights (not the biases); lossHistory [iterations]
 * (optional) gets the loss before each step. With a validation set (nVal > 0) its loss is
 * computed every evalEvery iterations (valHistory, optional, gets them) and the model
 * with the lowest validation loss is returned (early stopping). The mean and sd stay as
 * given. */
BIPP_B200_EXPORT BippError bipp_rank_mlp_train(bipp_ctx_t ctx, float* model, const float* features,
                                               const float* targets, size_t n, const float* valFeatures,
                                               const float* valTargets, size_t nVal, int iterations,
                                               float learningRate, float weightDecay, int evalEvery,
                                               float* lossHistory, float* valHistory);

/* Largest antenna count accepted by bipp_eigh_gram_noalloc_s. */
#define BIPP_NOALLOC_MAX_ANTENNA 128

/* No counterpart in the reference. eigh_gram for one time step (W = I, nBeam = nAntenna)
 * that allocates no device memory, for callers that cannot let a library call
 * cudaMalloc/cudaFree: an imager embedded in a host framework whose caching allocator
 * owns all device memory, or a real-time correlator loop that must not block on the
 * device-wide synchronisation of cudaFree. Intermediates live in one file-scope
 * __device__ array of about 1 MB, held by every GPU that loads the library until the
 * process exits; nAntenna above BIPP_NOALLOC_MAX_ANTENNA is rejected with
 * BIPP_INVALID_PARAMETER_ERROR. All pointers are DEVICE pointers owned by the caller:
 * s (nAntenna x nAntenna complex float, lower triangle used, lds), xyz (nAntenna x 3
 * double, ldxyz); outputs d[nAntenna] (ascending, zero padded), v (nAntenna x nAntenna,
 * ldv, zero padded), *nBeamReduced, *scale (= 1/nVis) and *info (1 if the Cholesky
 * factorisation of G failed, a kept entry of S is not finite or every row and column is
 * flagged, else 0). The call is asynchronous on `stream` (a
 * cudaStream_t). Every call on a device shares the array, so calls that overlap on the
 * GPU race; serialise them (one stream, or events). Each call makes `device` current while
 * it runs, gives the caller's current device back before it returns, and looks up the
 * array's address in that device's current context (cudaGetSymbolAddress, which allocates
 * nothing); the first call on a device may load the library's device code and should come
 * before any stream capture. Results agree with bipp_eigh_gram_s. */
BIPP_B200_EXPORT BippError bipp_eigh_gram_noalloc_s(int device, void* stream, float wl, size_t nAntenna,
                                                    const void* s, size_t lds, const double* xyz, size_t ldxyz,
                                                    float* d, void* v, size_t ldv, int* nBeamReduced, float* scale,
                                                    int* info);

/* Gram matrix G = W^H sinc(2|p_i - p_j| / wl) W, nBeam x nBeam complex; replaces
 * bipp::host::gram_matrix (src/host/gram_matrix.hpp:15-17). */
BIPP_B200_EXPORT BippError bipp_gram_matrix_s(bipp_ctx_t ctx, size_t nAntenna, size_t nBeam, const void* w,
                                              size_t ldw, const float* xyz, size_t ldxyz, float wl, void* g,
                                              size_t ldg);
BIPP_B200_EXPORT BippError bipp_gram_matrix_d(bipp_ctx_t ctx, size_t nAntenna, size_t nBeam, const void* w,
                                              size_t ldw, const double* xyz, size_t ldxyz, double wl, void* g,
                                              size_t ldg);

/* Virtual visibilities VV = V_k diag(scale d_k) V_k^H over the non-zero entries of d,
 * written as a column-major nAntenna x nAntenna matrix; replaces
 * bipp::host::virtual_vis (src/host/virtual_vis.hpp:15-17). */
BIPP_B200_EXPORT BippError bipp_virtual_vis_s(bipp_ctx_t ctx, float scale, size_t nAntenna, size_t nBeam,
                                              const float* d, const void* v, size_t ldv, void* vv);
BIPP_B200_EXPORT BippError bipp_virtual_vis_d(bipp_ctx_t ctx, double scale, size_t nAntenna, size_t nBeam,
                                              const double* d, const void* v, size_t ldv, void* vv);

/* Direct sum out[p] += Re sum_k input_k exp(i alpha (x_p u_k + y_p v_k + z_p w_k));
 * replaces bipp::host::nuft_sum / bipp::gpu::nuft_sum (src/host/kernels/nuft_sum.cpp:9-31,
 * src/gpu/kernels/nuft_sum.cu:24-84). The phase argument is formed and reduced in FP64;
 * the _s variant evaluates sine/cosine in FP32 on the reduced argument, _d in FP64. */
BIPP_B200_EXPORT BippError bipp_nuft_sum_s(bipp_ctx_t ctx, float alpha, size_t nIn, const void* input,
                                           const float* u, const float* v, const float* w, size_t nOut,
                                           const float* x, const float* y, const float* z, float* out);
BIPP_B200_EXPORT BippError bipp_nuft_sum_d(bipp_ctx_t ctx, double alpha, size_t nIn, const void* input,
                                           const double* u, const double* v, const double* w, size_t nOut,
                                           const double* x, const double* y, const double* z, double* out);
/* Multi-channel direct sum on DEVICE pointers (FP64 coordinates and outputs, FP32 complex
 * values [nch][ldIn]): the GPU check used for large pixel subsets. */
BIPP_B200_EXPORT BippError bipp_nuft_sum_multi_device(bipp_ctx_t ctx, double alpha, size_t nIn, size_t nch,
                                                      const void* values, size_t ldIn, const double* u,
                                                      const double* v, const double* w, size_t nOut,
                                                      const double* x, const double* y, const double* z,
                                                      double* out, size_t ldOut, int fp64Trig);

/* Bucket partition of points into a regular grid of groups; replaces
 * DomainPartition::grid (src/host/domain_partition.hpp:35-101). permut[i] is the sorted
 * position of point i; groupBegin/groupSize have dims[0]*dims[1]*dims[2] entries. A grid of
 * one group returns the identity (DomainPartition::none). */
BIPP_B200_EXPORT BippError bipp_domain_partition_grid_s(bipp_ctx_t ctx, const size_t* dims, size_t n,
                                                        const float* x, const float* y, const float* z,
                                                        size_t* permut, size_t* groupBegin, size_t* groupSize);
BIPP_B200_EXPORT BippError bipp_domain_partition_grid_d(bipp_ctx_t ctx, const size_t* dims, size_t n,
                                                        const double* x, const double* y, const double* z,
                                                        size_t* permut, size_t* groupBegin, size_t* groupSize);

/* ---- NUFFT synthesis: collect / get ---------------------------------------------------- */

/* Mirrors NufftSynthesisOptions and Partition (include/bipp/image_synthesis.hpp:23-148). */
typedef struct {
  int precision;            /* BippPrecision */
  float tolerance;          /* NUFFT tolerance */
  size_t sampleBatchSize;   /* 0 = automatic */
  int partitionMethod;      /* 0 = Auto, 1 = None, 2 = Grid */
  size_t partitionGrid[3];  /* Grid dimensions (u, v, w) */
  int normalizeImage;       /* divide by the number of samples */
  int applyScaling;         /* accepted; scale is always applied, as in the reference */
} bipp_nufft_options;

/* Create a collector for nImages images over nPixel output points (lmn: nPixel x 3,
 * FP32 as the ImageProp interface provides) and nBaselines points per added sample;
 * replaces gpu::NUFFT (src/gpu/nufft.hpp:31-62). */
BIPP_B200_EXPORT BippError bipp_nufft_create(bipp_ctx_t ctx, const bipp_nufft_options* opt, size_t nPixel,
                                             const float* lmn, size_t ldlmn, size_t nImages, size_t nBaselines,
                                             bipp_nufft_t* plan);
/* Append one sample: uvw nBaselines x 3 already scaled by 2 pi / wl (as the reference's
 * add, src/nufft_interface.hpp:16), values nBaselines x nImages complex. */
BIPP_B200_EXPORT BippError bipp_nufft_add_s(bipp_nufft_t plan, const float* uvw, size_t lduvw, const void* values,
                                            size_t ldvalues);
BIPP_B200_EXPORT BippError bipp_nufft_add_d(bipp_nufft_t plan, const double* uvw, size_t lduvw,
                                            const void* values, size_t ldvalues);
/* Transform what was collected and return image imgIdx (nPixel floats, accumulated real
 * part); src/nufft_interface.hpp:18. */
BIPP_B200_EXPORT BippError bipp_nufft_get_image(bipp_nufft_t plan, size_t imgIdx, float* image);
BIPP_B200_EXPORT BippError bipp_nufft_destroy(bipp_nufft_t plan);

/* ---- image synthesis over a dataset -------------------------------------------------------- */

/* Dataset accessors (include/bipp/dataset.hpp:14-41), called on the host. */
typedef struct {
  void* user;
  size_t (*num_samples)(void* user);
  size_t (*num_antenna)(void* user);
  size_t (*num_beam)(void* user);
  void (*eig_vec)(void* user, size_t index, void* v, size_t ldv);      /* complex float */
  void (*eig_val)(void* user, size_t index, float* d);
  void (*uvw)(void* user, size_t index, float* uvw, size_t lduvw);     /* metres */
  float (*wl)(void* user, size_t index);
  float (*scale)(void* user, size_t index);
} bipp_dataset_callbacks;

/* image_synthesis (include/bipp/image_synthesis.hpp:160-163) for nImages selections that
 * share the same nSamples sample ids. sampleIds: [nImages][nSamples]; eigvals:
 * [nImages][nSamples] pointers to nBeam scaled eigenvalues; images: [nImages][nPixel]
 * output (written, not accumulated). Validation and normalisation follow
 * src/image_synthesis.cpp:36-69, 152-163. */
BIPP_B200_EXPORT BippError bipp_image_synthesis(bipp_ctx_t ctx, const bipp_nufft_options* opt,
                                                const bipp_dataset_callbacks* dataset, size_t nImages,
                                                size_t nSamples, const size_t* sampleIds,
                                                const float* const* eigvals, size_t nPixel, const float* lmn,
                                                size_t ldlmn, float* images);

/* ---- batched pipeline: S, positions -> eigensolve -> levels -> VV -> NUFFT images ----- */

typedef struct {
  size_t nAntenna;        /* antennas per step (W = I) */
  size_t nLevels;         /* energy levels, 1 to 8 */
  const double* intervals;/* [nLevels][2] (lo, hi) eigenvalue intervals, lo <= hi (else
                             BIPP_INVALID_PARAMETER_ERROR); +-inf allowed */
  int filter;             /* 0 lsq, 1 std, 2 sqrt, 3 inv, 4 inv_sqrt (python/bipp/filter.py) */
  double tolerance;       /* NUFFT tolerance */
  size_t gridA, gridB;    /* pixel lattice extents (a slow, b fast); nPixel = gridA * gridB */
  double lattice[6];      /* l0, m0, A_l, B_l, A_m, B_m: l = l0 + a A_l + b B_l, m = m0 + a A_m + b B_m */
  const double* pixelN;   /* [nPixel] n coordinate of each pixel (FP64) */
  const double* uvwBasis; /* [9] column-major 3x3 (columns U, V, W in the position frame) */
  size_t chunkSteps;      /* steps per eigensolver launch sequence (0 = 256) */
  size_t maxSteps;        /* maximum steps per process() call */
  int mode;               /* 0 batched (one NUFFT per call), 1 plain (one NUFFT per step and level) */
  int vvPrecision;        /* arithmetic of the virtual-visibility products VV = X diag(s) X^H
                             (src/host/virtual_vis.cpp:52-68): 0 3xTF32 and 1 BF16x3 (tensor
                             cores, split operands, FP32 accumulation), 2 FP32 (CUDA cores),
                             3 FP64 (CUDA cores; for precision studies) */
} bipp_pipeline_config;

BIPP_B200_EXPORT BippError bipp_pipeline_create(bipp_ctx_t ctx, const bipp_pipeline_config* cfg,
                                                bipp_pipeline_t* pipeline);
/* Process nSteps time steps: s [nSteps][nAntenna x nAntenna] complex float (lower triangle
 * used), xyz [nSteps][nAntenna][3] FP64 positions, wl [nSteps] FP64. onDevice != 0: the
 * three pointers are device pointers (s is read in place, not modified), else host
 * pointers (copied in by the call; of s only the lower triangle is copied, in blocks of
 * 64 columns from each block's diagonal row down). The steps' contributions are
 * accumulated into the images. Fails with BIPP_EIGENSOLVER_ERROR when a Gram matrix is
 * not positive definite or a kept entry of some S is not finite (as bipp_eigh_gram_s;
 * checked after the eigensolve, so a failing call adds nothing to the images in batched
 * mode, while plain mode keeps the steps before the failing one), and with
 * BIPP_GPU_ERROR when a tensor-core completion wait runs out (a GPU fault). */
BIPP_B200_EXPORT BippError bipp_pipeline_process(bipp_pipeline_t pl, size_t nSteps, const void* s,
                                                 const double* xyz, const double* wl, int onDevice);
/* Double-buffered host input: bipp_pipeline_stage copies a batch (host arrays as for
 * bipp_pipeline_process with onDevice 0; pinned memory lets the copy run asynchronously)
 * into one of two device slots on a stream of its own and returns at once;
 * bipp_pipeline_process_staged processes the oldest staged batch. Staging batch k + 1
 * before processing batch k overlaps its copy with batch k's work. At most two batches
 * wait (BIPP_INVALID_PARAMETER_ERROR otherwise); the host arrays must stay unchanged until
 * the batch is processed. */
BIPP_B200_EXPORT BippError bipp_pipeline_stage(bipp_pipeline_t pl, size_t nSteps, const void* s, const double* xyz,
                                               const double* wl);
BIPP_B200_EXPORT BippError bipp_pipeline_process_staged(bipp_pipeline_t pl);
/* Images [nLevels][nPixel] (normalised by the number of processed steps if normalize),
 * to host (onDevice == 0) or device memory. */
BIPP_B200_EXPORT BippError bipp_pipeline_images(bipp_pipeline_t pl, float* images, int normalize, int onDevice);
BIPP_B200_EXPORT BippError bipp_pipeline_reset(bipp_pipeline_t pl);
/* Eigenvalues [maxSteps][nAntenna] and nBeamReduced of the last process() call (host).
 * Only the eigenvalues inside [min lo, max hi] of the energy levels are computed by the
 * pipeline (the others do not enter the images); the other entries are zero. */
BIPP_B200_EXPORT BippError bipp_pipeline_last_eigenvalues(bipp_pipeline_t pl, double* d, int* nReduced);
/* Accumulated device time (ms) per stage since the last reset (7 values): [0] eigensolver,
 * [1] virtual visibilities, [2] NUFFT point preparation and sort, [3] spreading kernel,
 * [4] FFT, [5] w-sum, [6] clearing of the fine-grid slabs. Only filled when timing is
 * enabled. */
BIPP_B200_EXPORT BippError bipp_pipeline_stage_times(bipp_pipeline_t pl, int enable, double* ms);
/* Accumulated device time (ms) of the eigensolver kernels since the last reset, when
 * timing is enabled: [0] flagging/compaction/Gram, [1] FP64 Cholesky, [2] triangular
 * inverse, [3] reduction GEMMs, [4] Householder tridiagonalisation, [5] tridiagonal
 * eigenpairs, [6] back-transform, [7] Linv^H Y GEMM. */
BIPP_B200_EXPORT BippError bipp_pipeline_kernel_times(bipp_pipeline_t pl, double* ms);
/* Statistics of the last NUFFT of the pipeline (9 values): points spread, spreading
 * launches (w-slabs), grid bytes written by the spreading, spreading work items, fine
 * grid sizes nx, ny, nw, kernel width W, tiles split into several work items (more points
 * than the spread.items_cap tuning parameter, 2048 by default; their parts accumulate into
 * the grid with atomics). */
BIPP_B200_EXPORT BippError bipp_pipeline_nufft_stats(bipp_pipeline_t pl, long long* stats);
BIPP_B200_EXPORT BippError bipp_pipeline_destroy(bipp_pipeline_t pl);

/* Self-test of the bounded tensor-core barrier waits (no counterpart in the reference):
 * waits with the given spin limit (1 to 2^20) on a barrier that nothing completes; the
 * wait gives up, *timedOut is set to 1 and the call fails with BIPP_GPU_ERROR, the way a
 * stuck MMA reaches the caller; the context stays usable. */
BIPP_B200_EXPORT BippError bipp_selftest_wait_timeout(bipp_ctx_t ctx, int spins, int* timedOut);

/* ---- autotuner of launch shapes (no counterpart in the reference, whose only launch-shape
 * logic is the fixed block-size ladder of src/gpu/kernels/nuft_sum.cu:73-84) ------------ */

/* Time the candidates of the tunable launch parameters on the caller's sample steps (the
 * arguments of bipp_pipeline_process) with the pipeline `pl`, one parameter at a time
 * (the pipeline's parameters of the tuning table below: spreading work items, A-operand
 * place, stages, CTAs per SM and schedule, threads and persistent CTAs of the
 * tridiagonalisation, virtual-visibility CTAs per SM). The time of a candidate is the
 * device time of the stage the parameter changes (spreading with tile clearing, the
 * tridiagonalisation kernel, or the virtual visibilities): every candidate gets one
 * untimed call, then max(2, repeats) passes over the candidates, forwards and backwards
 * in turn, and the fastest call of each counts. The fastest candidate of each parameter
 * is kept in the process-wide tuning table, unless the whole call with the tuned set is
 * slower than with the starting values (a value can speed up its own stage and slow the
 * call down elsewhere; both sets timed twice, interleaved), in which case the starting
 * values come back. A JSON report of those times (ms, and "whole_call_ms") is written
 * into report (reportLen bytes, truncated). The pipeline's images and step count
 * are left as they were. Results do not depend on the chosen values beyond rounding. */
BIPP_B200_EXPORT BippError bipp_autotune_pipeline(bipp_pipeline_t pl, size_t nSteps, const void* s, const double* xyz,
                                                  const double* wl, int onDevice, int repeats, char* report,
                                                  size_t reportLen);
/* The tuning table: get or set one parameter (a value outside its candidates fails with
 * BIPP_INVALID_PARAMETER_ERROR), describe all (one line each: name, value, candidates,
 * meaning), save to or load from a file of "name value" lines, or reset to the defaults.
 * BIPP_B200_TUNING_FILE, when set, is loaded on first use. No device is needed. */
BIPP_B200_EXPORT BippError bipp_tuning_get(const char* name, int* value);
BIPP_B200_EXPORT BippError bipp_tuning_set(const char* name, int value);
BIPP_B200_EXPORT BippError bipp_tuning_describe(char* out, size_t len);
BIPP_B200_EXPORT BippError bipp_tuning_save(const char* path);
BIPP_B200_EXPORT BippError bipp_tuning_load(const char* path);
BIPP_B200_EXPORT BippError bipp_tuning_reset(void);

#ifdef __cplusplus
}
#endif
