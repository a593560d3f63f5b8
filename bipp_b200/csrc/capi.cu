// C-ABI: context, error reporting, domain partition, dataset-driven image synthesis.
#include <algorithm>
#include <atomic>
#include <complex>
#include <cstring>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "context.hpp"
#include "eig_kernels.cuh"
#include "nufft.hpp"

// float/double multiply without contraction (reference arithmetic is a plain product)
template <typename T> __device__ __forceinline__ T fmul_rn_t(T a, T b);
template <> __device__ __forceinline__ float fmul_rn_t<float>(float a, float b) { return __fmul_rn(a, b); }
template <> __device__ __forceinline__ double fmul_rn_t<double>(double a, double b) { return __dmul_rn(a, b); }

namespace bippb200 {

// Message of the last failure on this thread. A plain character array: a thread_local
// std::string would be destroyed before objects with static storage duration, and a
// caller's static context released at exit still goes through guard().
static thread_local char g_lastError[1024];
static std::atomic<unsigned long long> g_launches{0};

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_last_error(const std::string& msg) {
  const size_t n = std::min(msg.size(), sizeof(g_lastError) - 1);
  std::memcpy(g_lastError, msg.data(), n);
  g_lastError[n] = '\0';
}

BippError guard(const std::function<void()>& body) {
  try {
    body();
    g_lastError[0] = '\0';
    return BIPP_SUCCESS;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_last_error("host allocation failed");
    return BIPP_GENERIC_ERROR;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return BIPP_GENERIC_ERROR;
  } catch (...) {
    set_last_error("unknown error");
    return BIPP_GENERIC_ERROR;
  }
}

// ---------------------------------------------------------------------------------------
// domain partition: group index per point, stable counting sort
// (src/host/domain_partition.hpp:35-101)
// ---------------------------------------------------------------------------------------
constexpr int kPartChunk = 4096;

template <typename T>
__global__ void part_group_kernel(long long n, const T* __restrict__ x, const T* __restrict__ y, const T* __restrict__ z,
                                  T minx, T miny, T minz, T invx, T invy, T invz, unsigned long long dx,
                                  unsigned long long dy, unsigned long long dz, int degx, int degy, int degz,
                                  unsigned long long* __restrict__ group) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    // same arithmetic as the reference: (size_t)(inv * (c - min)), clamped to dims - 1; on
    // an axis without extent the reference computes inf * 0 = NaN, whose conversion to
    // size_t on x86-64 lands in the last cell, so those points go to the last cell
    const T cx = fmul_rn_t(invx, (T)(x[i] - minx));
    const T cy = fmul_rn_t(invy, (T)(y[i] - miny));
    const T cz = fmul_rn_t(invz, (T)(z[i] - minz));
    unsigned long long gx = degx ? dx - 1 : (unsigned long long)cx;
    unsigned long long gy = degy ? dy - 1 : (unsigned long long)cy;
    unsigned long long gz = degz ? dz - 1 : (unsigned long long)cz;
    gx = gx < dx - 1 ? gx : dx - 1;
    gy = gy < dy - 1 ? gy : dy - 1;
    gz = gz < dz - 1 ? gz : dz - 1;
    group[i] = (gz * dy + gy) * dx + gx;
  }
}

__global__ void part_count_kernel(long long n, const unsigned long long* __restrict__ group, long long nChunks,
                                  int* __restrict__ counts) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long chunk = i / kPartChunk;
    atomicAdd(counts + group[i] * nChunks + chunk, 1);
  }
}

// one warp per chunk; points of the chunk are ranked in index order (stable)
__global__ void part_scatter_kernel(long long n, const unsigned long long* __restrict__ group, long long nChunks,
                                    int* __restrict__ cursor, unsigned long long* __restrict__ permut) {
  const long long chunk = blockIdx.x;
  const int lane = threadIdx.x;
  const long long beg = chunk * kPartChunk;
  const long long end = min(n, beg + kPartChunk);
  const unsigned lt = (1u << lane) - 1u;
  for (long long w0 = beg; w0 < end; w0 += 32) {
    const long long i = w0 + lane;
    const bool act = i < end;
    const unsigned long long key = act ? group[i] : ~0ull;
    const unsigned m = __match_any_sync(0xffffffffu, key);
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (act) base = cursor[key * nChunks + chunk];
    __syncwarp();
    if (act) permut[i] = (unsigned long long)(base + __popc(m & lt));
    __syncwarp();
    if (act && lane == leader) cursor[key * nChunks + chunk] = base + __popc(m);
    __syncwarp();
  }
}

template <typename T>
static void partition_host(bipp_ctx_s* ctx, const size_t* dims, size_t n, const T* x, const T* y, const T* z,
                           size_t* permut, size_t* gBegin, size_t* gSize) {
  require(dims && permut && gBegin && gSize, "null pointer", BIPP_INVALID_POINTER_ERROR);
  require(n == 0 || (x && y && z), "null pointer", BIPP_INVALID_POINTER_ERROR);
  const unsigned long long ng = (unsigned long long)dims[0] * dims[1] * dims[2];
  require(dims[0] > 0 && dims[1] > 0 && dims[2] > 0, "grid dimensions must be positive");
  if (ng <= 1 || n == 0) {
    for (size_t i = 0; i < n; ++i) permut[i] = i;
    if (ng >= 1) {
      gBegin[0] = 0;
      gSize[0] = n;
      for (unsigned long long g = 1; g < ng; ++g) { gBegin[g] = n; gSize[g] = 0; }
    }
    return;
  }
  const long long nChunks = ((long long)n + kPartChunk - 1) / kPartChunk;
  require(ng * (unsigned long long)nChunks < (1ull << 31), "partition grid too large for the point count");
  T mn[3], mx[3], inv[3];
  int deg[3];
  const T* c[3] = {x, y, z};
  for (int d = 0; d < 3; ++d) {
    auto mm = std::minmax_element(c[d], c[d] + n);
    mn[d] = *mm.first;
    mx[d] = *mm.second;
    inv[d] = T(dims[d]) / (mx[d] - mn[d]);
    deg[d] = !(mx[d] > mn[d]);
  }
  DevBuf dc(ctx, 3 * n * sizeof(T)), dg(ctx, n * sizeof(unsigned long long)), dp(ctx, n * sizeof(unsigned long long));
  const long long nc = (long long)ng * nChunks;
  DevBuf counts(ctx, (nc + 1) * sizeof(int)), offs(ctx, (nc + 1) * sizeof(int)), cursor(ctx, (nc + 1) * sizeof(int));
  const long long per = (long long)kScanThreads * kScanItems;
  const int nb = (int)((nc + per - 1) / per);
  DevBuf bs(ctx, (nb + 1) * sizeof(int));
  for (int d = 0; d < 3; ++d) h2d(ctx, dc.get<T>() + d * n, c[d], n * sizeof(T));
  counts.zero();
  const int blocks = (int)std::min<long long>(((long long)n + 255) / 256, 4096);
  count_launch();
  part_group_kernel<T><<<blocks, 256, 0, ctx->stream>>>((long long)n, dc.get<T>(), dc.get<T>() + n, dc.get<T>() + 2 * n,
                                                        mn[0], mn[1], mn[2], inv[0], inv[1], inv[2], dims[0], dims[1],
                                                        dims[2], deg[0], deg[1], deg[2], dg.get<unsigned long long>());
  count_launch();
  part_count_kernel<<<blocks, 256, 0, ctx->stream>>>((long long)n, dg.get<unsigned long long>(), nChunks, counts.get<int>());
  count_launch();
  scan_partial_kernel<<<nb, kScanThreads, 0, ctx->stream>>>(counts.get<int>(), offs.get<int>(), nc, bs.get<int>());
  count_launch();
  scan_blocksums_kernel<<<1, 1024, 0, ctx->stream>>>(bs.get<int>(), nb, offs.get<int>() + nc);
  count_launch();
  scan_add_kernel<<<nb, 1024, 0, ctx->stream>>>(offs.get<int>(), nc, bs.get<int>(), cursor.get<int>());
  count_launch();
  part_scatter_kernel<<<(int)nChunks, 32, 0, ctx->stream>>>((long long)n, dg.get<unsigned long long>(), nChunks,
                                                           cursor.get<int>(), dp.get<unsigned long long>());
  B2_CHECK_LAUNCH();
  std::vector<int> off(nc + 1);
  d2h(ctx, off.data(), offs.get(), (nc + 1) * sizeof(int));
  static_assert(sizeof(size_t) == sizeof(unsigned long long), "size_t must be 64-bit");
  d2h(ctx, permut, dp.get(), n * sizeof(unsigned long long));
  sync(ctx);
  for (unsigned long long g = 0; g < ng; ++g) {
    gBegin[g] = (size_t)off[g * nChunks];
    gSize[g] = (size_t)(off[(g + 1) * nChunks] - off[g * nChunks]);
  }
}

}  // namespace bippb200

using namespace bippb200;

namespace bippb200 {
// Pinned host slots for staged copies, each with an event recorded after the last copy
// that reads it
class PinnedSlots {
public:
  PinnedSlots(int n, size_t bytes) : bufs_(n, nullptr), events_(n, nullptr), recorded_(n, false) {
    for (int i = 0; i < n; ++i) {
      B2_CUDA(cudaMallocHost(&bufs_[i], bytes));
      B2_CUDA(cudaEventCreateWithFlags(&events_[i], cudaEventDisableTiming));
    }
  }
  PinnedSlots(const PinnedSlots&) = delete;
  PinnedSlots& operator=(const PinnedSlots&) = delete;
  ~PinnedSlots() {
    for (size_t i = 0; i < bufs_.size(); ++i) {
      if (events_[i]) {
        cudaEventSynchronize(events_[i]);
        cudaEventDestroy(events_[i]);
      }
      if (bufs_[i]) cudaFreeHost(bufs_[i]);
    }
  }
  void* get(int i) const { return bufs_[i]; }
  void record(int i, cudaStream_t st) {
    B2_CUDA(cudaEventRecord(events_[i], st));
    recorded_[i] = true;
  }
  void wait(int i) {
    if (recorded_[i]) B2_CUDA(cudaEventSynchronize(events_[i]));
  }

private:
  std::vector<void*> bufs_;
  std::vector<cudaEvent_t> events_;
  std::vector<bool> recorded_;
};

void ctx_release(bipp_ctx_s* c) {
  if (c->refs.fetch_sub(1) != 1) return;
  cudaStreamSynchronize(c->stream);
  cudaStreamDestroy(c->stream);
  delete c;
}
}  // namespace bippb200

extern "C" {

const char* bipp_last_error(void) { return g_lastError; }

unsigned long long bipp_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

BippError bipp_ctx_create_on_device(BippProcessingUnit pu, int device, bipp_ctx_t* out) {
  return guard([&] {
    require(out != nullptr, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(pu != BIPP_PU_CPU, "this library has no CPU processing unit; use BIPP_PU_GPU or BIPP_PU_AUTO");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw Error(BIPP_GPU_SUPPORT_ERROR, "no CUDA device available");
    }
    require(device >= 0 && device < count, "invalid device id");
    auto c = std::make_unique<bipp_ctx_s>();
    c->device = device;
    B2_CUDA(cudaSetDevice(device));
    B2_CUDA(cudaGetDeviceProperties(&c->prop, device));
    require(c->prop.major >= 10, "this library is built for sm_100a (B200) devices", BIPP_GPU_SUPPORT_ERROR);
    c->smCount = c->prop.multiProcessorCount;
    c->maxSmemOptin = c->prop.sharedMemPerBlockOptin;
    B2_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    // keep freed pool memory cached between calls
    cudaMemPool_t pool;
    B2_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
    unsigned long long thr = ~0ull;
    B2_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    *out = c.release();
  });
}

BippError bipp_ctx_create(BippProcessingUnit pu, bipp_ctx_t* out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    dev = 0;
  }
  return bipp_ctx_create_on_device(pu, dev, out);
}

BippError bipp_ctx_destroy(bipp_ctx_t ctx) {
  return guard([&] {
    if (!ctx) return;
    ctx_release(ctx);
  });
}

BippError bipp_ctx_processing_unit(bipp_ctx_t ctx, BippProcessingUnit* pu) {
  return guard([&] {
    require(ctx && pu, "null pointer", BIPP_INVALID_POINTER_ERROR);
    *pu = BIPP_PU_GPU;
  });
}

BippError bipp_ctx_stream(bipp_ctx_t ctx, void** stream) {
  return guard([&] {
    require(ctx && stream, "null pointer", BIPP_INVALID_POINTER_ERROR);
    *stream = (void*)ctx->stream;
  });
}

BippError bipp_domain_partition_grid_s(bipp_ctx_t ctx, const size_t* dims, size_t n, const float* x, const float* y,
                                       const float* z, size_t* permut, size_t* groupBegin, size_t* groupSize) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    partition_host<float>(ctx, dims, n, x, y, z, permut, groupBegin, groupSize);
  });
}
BippError bipp_domain_partition_grid_d(bipp_ctx_t ctx, const size_t* dims, size_t n, const double* x, const double* y,
                                       const double* z, size_t* permut, size_t* groupBegin, size_t* groupSize) {
  return guard([&] {
    require(ctx != nullptr, "null context", BIPP_INVALID_HANDLE_ERROR);
    partition_host<double>(ctx, dims, n, x, y, z, permut, groupBegin, groupSize);
  });
}

// image_synthesis over a callback dataset: validation (src/image_synthesis.cpp:36-69),
// per-sample uvw scaling by 2 pi / wl (src/nufft_synthesis.cpp:149-155), virtual
// visibilities of all images of a sample (src/nufft_synthesis.cpp:157-162) by one GPU
// launch per group of four images, written straight into the collectors' device staging
// buffers (no device-host round trip), collect/get NUFFT, normalisation by the number of
// samples (src/image_synthesis.cpp:152-163).
BippError bipp_image_synthesis(bipp_ctx_t ctx, const bipp_nufft_options* opt, const bipp_dataset_callbacks* ds,
                               size_t nImages, size_t nSamples, const size_t* sampleIds, const float* const* eigvals,
                               size_t nPixel, const float* lmn, size_t ldlmn, float* images) {
  return guard([&] {
    require(ctx && opt && ds && sampleIds && eigvals && lmn && images, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(nImages > 0, "Empty selection", BIPP_INVALID_PARAMETER_ERROR);
    require(nSamples > 0, "Empty selection", BIPP_INVALID_PARAMETER_ERROR);
    const size_t nTotal = ds->num_samples(ds->user);
    const size_t nAnt = ds->num_antenna(ds->user), nBeam = ds->num_beam(ds->user);
    // per image: sort by sample id, reject duplicates / out of range, ids must agree
    std::vector<std::vector<size_t>> order(nImages);
    for (size_t im = 0; im < nImages; ++im) {
      auto& o = order[im];
      o.resize(nSamples);
      std::iota(o.begin(), o.end(), 0);
      const size_t* ids = sampleIds + im * nSamples;
      std::stable_sort(o.begin(), o.end(), [&](size_t a, size_t b) { return ids[a] < ids[b]; });
      for (size_t k = 1; k < nSamples; ++k)
        require(ids[o[k]] != ids[o[k - 1]], "Selection sample id duplicate");
      require(ids[o[nSamples - 1]] < nTotal, "Selection sample id exceeds number of dataset samples");
    }
    for (size_t im = 1; im < nImages; ++im)
      for (size_t k = 0; k < nSamples; ++k)
        require(sampleIds[im * nSamples + order[im][k]] == sampleIds[order[0][k]],
                "Selection must contain the same sample ids for all images.");
    const size_t nB = nAnt * nAnt;
    // Samples are read into two pinned host slots; sample k + 1 is read (dataset callbacks)
    // while the copies and kernels of sample k run, and a slot is rewritten only after the
    // copies that read it have completed (its event). Eigenvectors and column scales go to
    // two device slots as well; the uvw go straight into the collectors' staging buffers.
    PinnedSlots host(2, nAnt * nBeam * sizeof(float2) + nB * 3 * sizeof(float) + nImages * nBeam * sizeof(float));
    DevBuf dV[2] = {DevBuf(ctx, nAnt * nBeam * sizeof(float2)), DevBuf(ctx, nAnt * nBeam * sizeof(float2))};
    DevBuf dK[2] = {DevBuf(ctx, nImages * nBeam * sizeof(float)), DevBuf(ctx, nImages * nBeam * sizeof(float))};
    DevBuf dn(ctx, 3 * 4 * sizeof(int));
    std::vector<int> hn(12);
    for (int i = 0; i < 4; ++i) {
      hn[i] = (int)nAnt;          // matrix size of every image of a group
      hn[4 + i] = 0;              // first column
      hn[8 + i] = (int)nBeam;     // end column
    }
    h2d(ctx, dn.get(), hn.data(), hn.size() * sizeof(int));
    // collectors in groups of 4 images
    std::vector<bipp_nufft_t> plans;
    for (size_t g0 = 0; g0 < nImages; g0 += 4) {
      bipp_nufft_options o = *opt;
      if (o.sampleBatchSize == 0) o.sampleBatchSize = std::min<size_t>(std::max<size_t>(1, 2000000000ull / (20 * nB)), nSamples);
      bipp_nufft_t p = nullptr;
      const BippError e = bipp_nufft_create(ctx, &o, nPixel, lmn, ldlmn, std::min<size_t>(4, nImages - g0), nB, &p);
      if (e != BIPP_SUCCESS) {
        for (auto q : plans) bipp_nufft_destroy(q);
        throw Error(e, bipp_last_error());
      }
      plans.push_back(p);
    }
    struct Cleanup {
      std::vector<bipp_nufft_t>& p;
      ~Cleanup() { for (auto q : p) bipp_nufft_destroy(q); }
    } cleanup{plans};
    // 2 pi rounded to float, as the reference's T(2 * pi) with T = float
    const float twoPi = static_cast<float>(2.0 * 3.14159265358979323846);
    for (size_t k = 0; k < nSamples; ++k) {
      const int slot = (int)(k & 1);
      host.wait(slot);   // the copies of sample k - 2 out of this slot are done
      auto* v = reinterpret_cast<std::complex<float>*>(host.get(slot));
      float* uvw = reinterpret_cast<float*>(v + nAnt * nBeam);
      float* ks = uvw + nB * 3;
      const size_t id = sampleIds[order[0][k]];
      const float wl = ds->wl(ds->user, id);
      const float scale = ds->scale(ds->user, id);
      ds->uvw(ds->user, id, uvw, nB);
      ds->eig_vec(ds->user, id, v, nAnt);
      // uvw scaled in single precision as the reference's float path
      const float uvwScale = twoPi / wl;   // float division (src/nufft_synthesis.cpp:150-154)
      for (size_t i = 0; i < nB * 3; ++i) uvw[i] *= uvwScale;
      for (size_t im = 0; im < nImages; ++im) {
        const float* d = eigvals[im * nSamples + order[im][k]];
        for (size_t c = 0; c < nBeam; ++c) ks[im * nBeam + c] = scale * d[c];
      }
      h2d(ctx, dV[slot].get(), v, nAnt * nBeam * sizeof(float2));
      h2d(ctx, dK[slot].get(), ks, nImages * nBeam * sizeof(float));
      for (size_t g0 = 0, gi = 0; g0 < nImages; g0 += 4, ++gi) {
        bipp_nufft_t pl = plans[gi];
        const long long ld = nufft_stage_ld(pl);
        float* su = nufft_stage_uvw(pl);
        for (int c = 0; c < 3; ++c) h2d(ctx, su + c * ld, uvw + c * nB, nB * sizeof(float));
        if (g0 + 4 >= nImages) host.record(slot, ctx->stream);   // last reader of the slot
        // VV of the group's images in one launch: "matrix" b = image g0 + b, the same
        // eigenvectors, its own column scales, output into the image's staging slot
        const int nIm = (int)std::min<size_t>(4, nImages - g0);
        GemmArgs<float2> g{};
        g.A = dV[slot].get<float2>(); g.strideA = 0; g.lda = (int)nAnt; g.opA = 0;
        g.B = dV[slot].get<float2>(); g.strideB = 0; g.ldb = (int)nAnt; g.opB = 1;
        g.Cm = nufft_stage_values(pl, 0); g.strideC = ld; g.ldc = (int)nAnt;
        g.n = dn.get<int>(); g.outMode = 0; g.levels = 1;
        g.kscale = dK[slot].get<float>() + g0 * nBeam; g.strideK = (long long)nBeam;
        g.kbeg = dn.get<int>() + 4; g.kend = dn.get<int>() + 8;
        const int tiles = ((int)nAnt + kGemmBM - 1) / kGemmBM;
        count_launch();
        gemm_kernel<float2, float><<<dim3(tiles, tiles, nIm), kGemmThreads, 0, ctx->stream>>>(g);
        B2_CHECK_LAUNCH();
        nufft_commit(pl);
      }
    }
    sync(ctx);
    for (size_t im = 0; im < nImages; ++im) {
      const BippError e = bipp_nufft_get_image(plans[im / 4], im % 4, images + im * nPixel);
      if (e != BIPP_SUCCESS) throw Error(e, bipp_last_error());
    }
    if (opt->normalizeImage) {
      const float s = 1.f / float(nSamples);
      for (size_t i = 0; i < nImages * nPixel; ++i) images[i] *= s;
    }
  });
}

}  // extern "C"
