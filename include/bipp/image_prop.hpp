// Abstract image properties (reference: include/bipp/image_prop.hpp:16-33).
#pragma once

#include <bipp/config.h>

#include <cstddef>
#include <string>
#include <unordered_map>
#include <variant>
#include <vector>

namespace bipp {

class BIPP_EXPORT ImageProp {
public:
  using MetaType = std::variant<std::size_t, float, std::vector<float>>;
  virtual void pixel_lmn(float* lmn, std::size_t ldlmn) = 0;
  virtual std::unordered_map<std::string, MetaType> meta_data() const = 0;
  virtual void set_meta(const std::string& name, const MetaType& data) = 0;
  virtual std::size_t width() const = 0;
  virtual std::size_t height() const = 0;
  virtual float fov_deg() const = 0;
  virtual ~ImageProp() = default;
};

}  // namespace bipp
