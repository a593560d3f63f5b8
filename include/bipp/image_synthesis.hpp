// Image synthesis of the bipp C++ API (reference: include/bipp/image_synthesis.hpp:23-163)
// plus the public collect/get synthesis object that the reference keeps internal
// (src/nufft_interface.hpp:13-21).
#pragma once

#include <bipp/config.h>
#include <bipp/context.hpp>
#include <bipp/dataset.hpp>
#include <bipp/enums.h>
#include <bipp/image_data.hpp>
#include <bipp/image_prop.hpp>

#include <array>
#include <complex>
#include <cstddef>
#include <memory>
#include <optional>
#include <string>
#include <unordered_map>
#include <utility>
#include <variant>
#include <vector>

namespace bipp {

struct Partition {
  Partition() = default;
  struct Auto {};
  struct None {};
  struct Grid {
    std::array<std::size_t, 3> dimensions = {1, 1, 1};
  };
  Partition(Partition::Grid g) : method(std::move(g)) {}
  Partition(Partition::Auto g) : method(std::move(g)) {}
  Partition(Partition::None g) : method(std::move(g)) {}
  std::variant<Partition::Auto, Partition::None, Partition::Grid> method = Partition::Auto();
};

struct NufftSynthesisOptions {
  BippPrecision precision = BIPP_PRECISION_SINGLE;
  float tolerance = 0.001f;
  std::optional<std::size_t> sampleBatchSize = std::nullopt;
  Partition localUVWPartition = Partition{Partition::Auto()};
  bool normalizeImage = true;
  bool apply_scaling = true;

  inline auto set_tolerance(float tol) -> NufftSynthesisOptions& { tolerance = tol; return *this; }
  inline auto set_sample_batch_size(std::optional<std::size_t> size) -> NufftSynthesisOptions& {
    sampleBatchSize = size;
    return *this;
  }
  inline auto set_local_uvw_partition(Partition p) -> NufftSynthesisOptions& {
    localUVWPartition = std::move(p);
    return *this;
  }
  inline auto set_normalize_image(bool normalize) -> NufftSynthesisOptions& { normalizeImage = normalize; return *this; }
  inline auto set_apply_scaling(bool apply) -> NufftSynthesisOptions& { apply_scaling = apply; return *this; }
  inline auto set_precision(BippPrecision prec) -> NufftSynthesisOptions& { precision = prec; return *this; }
};

using Selection = std::unordered_map<std::string, std::vector<std::pair<std::size_t, const float*>>>;

// Image synthesis into an ImageData object (one image per selection tag).
BIPP_EXPORT void image_synthesis(Context& ctx, const NufftSynthesisOptions& opt, Dataset& dataset, Selection selection,
                                 ImageProp& imageProp, ImageData& imageData);

// The reference's signature, writing an image file. This build has no HDF5: the call
// throws HDF5Error; use the ImageData overload.
BIPP_EXPORT void image_synthesis(Context& ctx, const NufftSynthesisOptions& opt, Dataset& dataset, Selection selection,
                                 ImageProp& imageProp, const std::string& imageFileName);

// Collect/get synthesis (NUFFTInterface::add / get_image): add samples of nBaselines
// points (uvw scaled by 2 pi / wl) with one complex value per image, then read images.
template <typename T>
class BIPP_EXPORT NufftSynthesis {
public:
  NufftSynthesis(Context& ctx, const NufftSynthesisOptions& opt, std::size_t nPixel, const float* lmn,
                 std::size_t ldlmn, std::size_t nImages, std::size_t nBaselines);
  void add(const T* uvw, std::size_t lduvw, const std::complex<T>* values, std::size_t ldvalues);
  void get_image(std::size_t imgIdx, float* image);
  ~NufftSynthesis();

private:
  struct Impl;
  std::unique_ptr<Impl> impl_;
};

}  // namespace bipp
