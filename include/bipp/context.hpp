// Context of the bipp C++ API (reference: include/bipp/context.hpp:17-76). Owns one GPU
// context of the B200 library (device = rank % device count, as the reference).
#pragma once

#include <bipp/communicator.hpp>
#include <bipp/config.h>
#include <bipp/enums.h>

#include <memory>

namespace bipp {

class ContextInternal;
struct InternalContextAccessor;

class BIPP_EXPORT Context {
public:
  explicit Context(BippProcessingUnit pu);
  Context(BippProcessingUnit pu, Communicator comm);
  Context(Context&&) = default;
  Context(const Context&) = delete;
  Context& operator=(Context&&) = default;
  Context& operator=(const Context&) = delete;

  auto processing_unit() const -> BippProcessingUnit;
  auto communicator() const -> const Communicator&;

private:
  friend InternalContextAccessor;
  std::shared_ptr<ContextInternal> ctx_;
  Communicator comm_;
};

}  // namespace bipp
