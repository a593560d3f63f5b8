// Communicator of the bipp C++ API (reference: include/bipp/communicator.hpp:22-89).
// This build has no MPI: world() describes the process group launched around the
// program through the RANK / WORLD_SIZE environment variables (one process per GPU);
// image reduction across ranks is done by the caller's collective library.
#pragma once

#include <bipp/config.h>

#include <cstddef>

namespace bipp {

class BIPP_EXPORT Communicator {
public:
  static auto world() -> Communicator;
  static auto local() -> Communicator;
  inline auto rank() const -> std::size_t { return rank_; }
  inline auto size() const -> std::size_t { return size_; }

private:
  Communicator() = default;
  std::size_t rank_ = 0;
  std::size_t size_ = 1;
};

}  // namespace bipp
