// The bipp C++ API (include/bipp/*.hpp) implemented over the C ABI of this library.
#include <algorithm>
#include <complex>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "bipp/bipp.hpp"
#include "bipp_b200.h"

namespace bippb200 {
void tcp_reduce_sum_to_root(const char* host, int port, std::size_t rank, std::size_t size, float* data,
                            std::size_t count, double timeoutSec);
}  // namespace bippb200

namespace bipp {

[[noreturn]] static void throw_code(BippError code) {
  const std::string msg = bipp_last_error();
  switch (code) {
    case BIPP_INTERNAL_ERROR: throw InternalError(msg);
    case BIPP_INVALID_PARAMETER_ERROR: throw InvalidParameterError(msg);
    case BIPP_INVALID_POINTER_ERROR: throw InvalidPointerError(msg);
    case BIPP_EIGENSOLVER_ERROR: throw EigensolverError(msg);
    case BIPP_NOT_IMPLEMENTED_ERROR: throw NotImplementedError(msg);
    case BIPP_GPU_ERROR: throw GPUError(msg);
    case BIPP_GPU_SUPPORT_ERROR: throw GPUSupportError(msg);
    case BIPP_GPU_BLAS_ERROR: throw GPUBlasError(msg);
    case BIPP_HDF5_ERROR: throw HDF5Error(msg);
    case BIPP_FILE_ERROR: throw FileError(msg);
    default: throw GenericError(msg);
  }
}

static void check(BippError code) {
  if (code != BIPP_SUCCESS) throw_code(code);
}

// ---- communicator / context ------------------------------------------------------------

auto Communicator::world() -> Communicator {
  Communicator c;
  const char* r = std::getenv("RANK");
  const char* s = std::getenv("WORLD_SIZE");
  c.rank_ = r ? std::strtoull(r, nullptr, 10) : 0;
  c.size_ = s ? std::max<std::size_t>(1, std::strtoull(s, nullptr, 10)) : 1;
  if (c.rank_ >= c.size_) throw InvalidParameterError("RANK must be below WORLD_SIZE");
  if (c.size_ > 1) {
    // images are summed into rank 0 over TCP, on MASTER_ADDR and a port of its own
    const char* host = std::getenv("MASTER_ADDR");
    const char* rp = std::getenv("BIPP_B200_REDUCE_PORT");
    const char* mp = std::getenv("MASTER_PORT");
    const char* to = std::getenv("BIPP_B200_REDUCE_TIMEOUT");
    const std::string h = (host && *host) ? host : "127.0.0.1";
    const int port = (rp && *rp) ? std::atoi(rp) : (mp && *mp) ? std::atoi(mp) + 17 : -1;
    const double timeout = (to && *to) ? std::atof(to) : 300.0;
    const std::size_t rank = c.rank_, size = c.size_;
    c.reduce_ = [h, port, rank, size, timeout](float* data, std::size_t count) {
      if (port <= 0 || port > 65535)
        throw InvalidParameterError("set MASTER_PORT or BIPP_B200_REDUCE_PORT for the image reduction of world()");
      bippb200::tcp_reduce_sum_to_root(h.c_str(), port, rank, size, data, count, timeout);
    };
  }
  return c;
}

auto Communicator::local() -> Communicator { return Communicator(); }

auto Communicator::custom(std::size_t rank, std::size_t size, ReduceFn reduceSumToRoot) -> Communicator {
  if (size < 1 || rank >= size) throw InvalidParameterError("communicator rank must be below its size");
  if (size > 1 && !reduceSumToRoot) throw InvalidParameterError("a communicator of several ranks needs a reduction");
  Communicator c;
  c.rank_ = rank;
  c.size_ = size;
  c.reduce_ = std::move(reduceSumToRoot);
  return c;
}

void Communicator::reduce_sum_to_root(float* data, std::size_t count) const {
  if (size_ <= 1) return;
  if (!reduce_) throw InvalidParameterError("this communicator has no reduction");
  try {
    reduce_(data, count);
  } catch (const GenericError&) {
    throw;
  } catch (const std::exception& e) {
    throw GenericError(e.what());
  }
}

class ContextInternal {
public:
  ContextInternal(BippProcessingUnit pu, std::size_t rank) {
    // the processing unit is checked before the devices, as by the C ABI
    if (pu == BIPP_PU_CPU)
      throw InvalidParameterError("this library has no CPU processing unit; use BIPP_PU_GPU or BIPP_PU_AUTO");
    // device = rank % device count (src/context_internal.cpp:59-66)
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
      cudaGetLastError();
      throw GPUSupportError("no CUDA device available");
    }
    check(bipp_ctx_create_on_device(pu, (int)(rank % (std::size_t)count), &ctx));
  }
  ~ContextInternal() {
    if (ctx) bipp_ctx_destroy(ctx);
  }
  bipp_ctx_t ctx = nullptr;
};

struct InternalContextAccessor {
  static auto get(const Context& c) -> bipp_ctx_t { return c.ctx_->ctx; }
};

Context::Context(BippProcessingUnit pu) : ctx_(new ContextInternal(pu, 0)), comm_(Communicator::local()) {}

Context::Context(BippProcessingUnit pu, Communicator comm)
    : ctx_(new ContextInternal(pu, comm.rank())), comm_(std::move(comm)) {}

auto Context::processing_unit() const -> BippProcessingUnit {
  BippProcessingUnit pu = BIPP_PU_GPU;
  check(bipp_ctx_processing_unit(ctx_->ctx, &pu));
  return pu;
}

auto Context::communicator() const -> const Communicator& { return comm_; }

static bipp_ctx_t default_ctx() {
  static std::once_flag once;
  static std::unique_ptr<ContextInternal> ctx;
  std::call_once(once, [] { ctx.reset(new ContextInternal(BIPP_PU_AUTO, 0)); });
  return ctx->ctx;
}

// ---- eigensolvers -------------------------------------------------------------------------

template <typename T, typename>
auto eigh(T wl, std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* s, std::size_t lds,
          const std::complex<T>* w, std::size_t ldw, T* d, std::complex<T>* v, std::size_t ldv)
    -> std::pair<std::size_t, T> {
  std::size_t nred = 0;
  T scale = 0;
  if constexpr (std::is_same_v<T, float>)
    check(bipp_eigh_s(default_ctx(), wl, nAntenna, nBeam, s, lds, w, ldw, d, v, ldv, &nred, &scale));
  else
    check(bipp_eigh_d(default_ctx(), wl, nAntenna, nBeam, s, lds, w, ldw, d, v, ldv, &nred, &scale));
  return {nred, scale};
}

template <typename T, typename>
auto eigh_gram(T wl, std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* s, std::size_t lds,
               const std::complex<T>* w, std::size_t ldw, const T* xyz, std::size_t ldxyz, T* d, std::complex<T>* v,
               std::size_t ldv) -> std::pair<std::size_t, T> {
  std::size_t nred = 0;
  T scale = 0;
  if constexpr (std::is_same_v<T, float>)
    check(bipp_eigh_gram_s(default_ctx(), wl, nAntenna, nBeam, s, lds, w, ldw, xyz, ldxyz, d, v, ldv, &nred, &scale));
  else
    check(bipp_eigh_gram_d(default_ctx(), wl, nAntenna, nBeam, s, lds, w, ldw, xyz, ldxyz, d, v, ldv, &nred, &scale));
  return {nred, scale};
}

template BIPP_EXPORT auto eigh<float, void>(float, std::size_t, std::size_t, const std::complex<float>*, std::size_t,
                                            const std::complex<float>*, std::size_t, float*, std::complex<float>*,
                                            std::size_t) -> std::pair<std::size_t, float>;
template BIPP_EXPORT auto eigh<double, void>(double, std::size_t, std::size_t, const std::complex<double>*,
                                             std::size_t, const std::complex<double>*, std::size_t, double*,
                                             std::complex<double>*, std::size_t) -> std::pair<std::size_t, double>;
template BIPP_EXPORT auto eigh_gram<float, void>(float, std::size_t, std::size_t, const std::complex<float>*,
                                                 std::size_t, const std::complex<float>*, std::size_t, const float*,
                                                 std::size_t, float*, std::complex<float>*, std::size_t)
    -> std::pair<std::size_t, float>;
template BIPP_EXPORT auto eigh_gram<double, void>(double, std::size_t, std::size_t, const std::complex<double>*,
                                                  std::size_t, const std::complex<double>*, std::size_t, const double*,
                                                  std::size_t, double*, std::complex<double>*, std::size_t)
    -> std::pair<std::size_t, double>;

// ---- synthesis ----------------------------------------------------------------------------

static bipp_nufft_options to_c(const NufftSynthesisOptions& o) {
  bipp_nufft_options c{};
  c.precision = o.precision;
  c.tolerance = o.tolerance;
  c.sampleBatchSize = o.sampleBatchSize.value_or(0);
  c.partitionMethod = 0;
  c.partitionGrid[0] = c.partitionGrid[1] = c.partitionGrid[2] = 1;
  if (std::holds_alternative<Partition::None>(o.localUVWPartition.method)) c.partitionMethod = 1;
  if (auto* g = std::get_if<Partition::Grid>(&o.localUVWPartition.method)) {
    c.partitionMethod = 2;
    for (int i = 0; i < 3; ++i) c.partitionGrid[i] = g->dimensions[i];
  }
  c.normalizeImage = o.normalizeImage ? 1 : 0;
  c.applyScaling = o.apply_scaling ? 1 : 0;
  return c;
}

namespace {
struct DatasetThunk {
  static std::size_t num_samples(void* u) { return static_cast<Dataset*>(u)->num_samples(); }
  static std::size_t num_antenna(void* u) { return static_cast<Dataset*>(u)->num_antenna(); }
  static std::size_t num_beam(void* u) { return static_cast<Dataset*>(u)->num_beam(); }
  static void eig_vec(void* u, std::size_t i, void* v, std::size_t ldv) {
    static_cast<Dataset*>(u)->eig_vec(i, static_cast<std::complex<float>*>(v), ldv);
  }
  static void eig_val(void* u, std::size_t i, float* d) { static_cast<Dataset*>(u)->eig_val(i, d); }
  static void uvw(void* u, std::size_t i, float* x, std::size_t ld) { static_cast<Dataset*>(u)->uvw(i, x, ld); }
  static float wl(void* u, std::size_t i) { return static_cast<Dataset*>(u)->wl(i); }
  static float scale(void* u, std::size_t i) { return static_cast<Dataset*>(u)->scale(i); }
};
}  // namespace

void image_synthesis(Context& ctx, const NufftSynthesisOptions& opt, Dataset& dataset, Selection selection,
                     ImageProp& imageProp, ImageData& imageData) {
  // names must not contain '/', '.', ' ' (src/image_synthesis.cpp:36-47)
  std::vector<std::string> tags;
  for (auto& [name, samples] : selection) {
    if (name.find('/') != std::string::npos) throw InvalidParameterError("Selection name must not contain '/'");
    if (name.find('.') != std::string::npos) throw InvalidParameterError("Selection name must not contain '.'");
    if (name.find(' ') != std::string::npos) throw InvalidParameterError("Selection name must not contain spaces");
    if (samples.empty()) throw InvalidParameterError("Empty selection");
    tags.push_back(name);
  }
  if (tags.empty()) throw InvalidParameterError("Empty selection");
  const std::size_t nSamples = selection[tags[0]].size();
  const Communicator& comm = ctx.communicator();
  const std::size_t nRanks = comm.size(), rank = comm.rank();
  // several ranks: the selection is sorted by sample id and checked as a whole, then each
  // rank images a contiguous block of ceil(n / size) samples (src/image_synthesis.cpp:52-80;
  // a rank whose block starts past the end images none)
  if (nRanks > 1) {
    for (const auto& t : tags) {
      auto& smp = selection[t];
      std::sort(smp.begin(), smp.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
      if (std::adjacent_find(smp.begin(), smp.end(), [](const auto& a, const auto& b) { return a.first == b.first; }) !=
          smp.end())
        throw InvalidParameterError("Selection sample id duplicate");
      if (smp.back().first >= dataset.num_samples())
        throw InvalidParameterError("Selection sample id exceeds number of dataset samples");
      if (smp.size() != nSamples)
        throw InvalidParameterError("Selection must contain the same sample ids for all images.");
      for (std::size_t i = 0; i < nSamples; ++i)
        if (smp[i].first != selection[tags[0]][i].first)
          throw InvalidParameterError("Selection must contain the same sample ids for all images.");
    }
  }
  const std::size_t per = (nSamples + nRanks - 1) / nRanks;
  const std::size_t begin = std::min(nSamples, rank * per);
  const std::size_t nLocal = nRanks > 1 ? std::min(per, nSamples - begin) : nSamples;
  std::vector<std::size_t> ids;
  std::vector<const float*> ev;
  for (const auto& t : tags) {
    if (selection[t].size() != nSamples)
      throw InvalidParameterError("Selection must contain the same sample ids for all images.");
    for (std::size_t i = begin; i < begin + nLocal; ++i) {
      ids.push_back(selection[t][i].first);
      ev.push_back(selection[t][i].second);
    }
  }
  const std::size_t nPixel = imageProp.width() * imageProp.height();
  std::vector<float> lmn(nPixel * 3);
  imageProp.pixel_lmn(lmn.data(), nPixel);
  std::vector<float> images(tags.size() * nPixel, 0.f);
  bipp_dataset_callbacks cb{&dataset,         &DatasetThunk::num_samples, &DatasetThunk::num_antenna,
                            &DatasetThunk::num_beam, &DatasetThunk::eig_vec, &DatasetThunk::eig_val,
                            &DatasetThunk::uvw,      &DatasetThunk::wl,      &DatasetThunk::scale};
  bipp_nufft_options o = to_c(opt);
  if (nRanks > 1) o.normalizeImage = 0;   // normalised once, on rank 0, after the sum
  if (nLocal)
    check(bipp_image_synthesis(InternalContextAccessor::get(ctx), &o, &cb, tags.size(), nLocal, ids.data(), ev.data(),
                               nPixel, lmn.data(), nPixel, images.data()));
  if (nRanks > 1) {
    // SUM of the images into rank 0 (src/image_synthesis.cpp:140-147), normalised there by
    // the total number of samples (:152-163); only rank 0 writes the image
    comm.reduce_sum_to_root(images.data(), images.size());
    if (rank != 0) return;
    if (opt.normalizeImage) {
      const float sc = 1.f / (float)nSamples;
      for (float& x : images) x *= sc;
    }
  }
  for (std::size_t i = 0; i < tags.size(); ++i) imageData.set(tags[i], images.data() + i * nPixel);
}

void image_synthesis(Context&, const NufftSynthesisOptions&, Dataset&, Selection, ImageProp&, const std::string&) {
  throw HDF5Error("HDF5 image files are not available in this build; use the ImageData overload");
}

template <typename T>
struct NufftSynthesis<T>::Impl {
  std::vector<bipp_nufft_t> plans;
  std::size_t nImages = 0, nBaselines = 0;
  ~Impl() {
    for (auto p : plans) bipp_nufft_destroy(p);
  }
};

template <typename T>
NufftSynthesis<T>::NufftSynthesis(Context& ctx, const NufftSynthesisOptions& opt, std::size_t nPixel, const float* lmn,
                                  std::size_t ldlmn, std::size_t nImages, std::size_t nBaselines)
    : impl_(new Impl) {
  impl_->nImages = nImages;
  impl_->nBaselines = nBaselines;
  const bipp_nufft_options o = to_c(opt);
  for (std::size_t g = 0; g < nImages; g += 4) {
    bipp_nufft_t p = nullptr;
    check(bipp_nufft_create(InternalContextAccessor::get(ctx), &o, nPixel, lmn, ldlmn, std::min<std::size_t>(4, nImages - g),
                            nBaselines, &p));
    impl_->plans.push_back(p);
  }
}

template <typename T>
void NufftSynthesis<T>::add(const T* uvw, std::size_t lduvw, const std::complex<T>* values, std::size_t ldvalues) {
  for (std::size_t g = 0, i = 0; g < impl_->nImages; g += 4, ++i) {
    if constexpr (std::is_same_v<T, float>)
      check(bipp_nufft_add_s(impl_->plans[i], uvw, lduvw, values + g * ldvalues, ldvalues));
    else
      check(bipp_nufft_add_d(impl_->plans[i], uvw, lduvw, values + g * ldvalues, ldvalues));
  }
}

template <typename T>
void NufftSynthesis<T>::get_image(std::size_t imgIdx, float* image) {
  if (imgIdx >= impl_->nImages) throw InvalidParameterError("image index out of range");
  check(bipp_nufft_get_image(impl_->plans[imgIdx / 4], imgIdx % 4, image));
}

template <typename T>
NufftSynthesis<T>::~NufftSynthesis() = default;

template class BIPP_EXPORT NufftSynthesis<float>;
template class BIPP_EXPORT NufftSynthesis<double>;

}  // namespace bipp
