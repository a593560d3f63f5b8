// Communicator of the bipp C++ API (reference: include/bipp/communicator.hpp:22-89).
// This build has no MPI. world() describes the process group launched around the program
// through the RANK / WORLD_SIZE environment variables (one process per GPU) and reduces
// images over TCP to rank 0 (MASTER_ADDR, default 127.0.0.1, and a port from
// BIPP_B200_REDUCE_PORT or MASTER_PORT + 17). custom() takes the caller's own reduction
// (for instance an MPI_Reduce of its MPI communicator) in place of the reference's
// custom(MPI_Comm).
#pragma once

#include <bipp/config.h>

#include <cstddef>
#include <functional>

namespace bipp {

class BIPP_EXPORT Communicator {
public:
  // sum `count` floats of every rank into rank 0's `data` (other ranks' data unspecified
  // afterwards); called by every rank with the same count
  using ReduceFn = std::function<void(float* data, std::size_t count)>;

  static auto world() -> Communicator;
  static auto local() -> Communicator;
  static auto custom(std::size_t rank, std::size_t size, ReduceFn reduceSumToRoot) -> Communicator;
  inline auto rank() const -> std::size_t { return rank_; }
  inline auto size() const -> std::size_t { return size_; }
  // the sum-to-root reduction of this group (nothing to do for one rank)
  void reduce_sum_to_root(float* data, std::size_t count) const;

private:
  Communicator() = default;
  std::size_t rank_ = 0;
  std::size_t size_ = 1;
  ReduceFn reduce_;
};

}  // namespace bipp
