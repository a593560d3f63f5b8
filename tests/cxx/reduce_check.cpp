// Host-side check of the C++ API's image reduction (no GPU): every rank started with
// RANK / WORLD_SIZE / MASTER_ADDR / BIPP_B200_REDUCE_PORT sums its array into rank 0
// through Communicator::world(); rank 0 checks the exact sum. Then a custom() communicator
// whose reduction is the caller's function. Exits 0 when the checks hold.
#include <bipp/bipp.hpp>

#include <cstdio>
#include <cstdlib>
#include <vector>

int main() {
  const auto w = bipp::Communicator::world();
  std::vector<float> a(100000);
  for (std::size_t i = 0; i < a.size(); ++i) a[i] = (float)((w.rank() + 1) * (i % 1000 + 1));
  try {
    w.reduce_sum_to_root(a.data(), a.size());
  } catch (const bipp::GenericError& e) {
    std::fprintf(stderr, "reduction failed: %s\n", e.what());
    return 1;
  }
  if (w.rank() == 0) {
    const double ranks = (double)w.size() * (w.size() + 1) / 2;
    for (std::size_t i = 0; i < a.size(); ++i)
      if (a[i] != (float)(ranks * (i % 1000 + 1))) {
        std::fprintf(stderr, "wrong sum at %zu: %f\n", i, a[i]);
        return 1;
      }
  }
  // the caller's reduction
  int calls = 0;
  const auto c = bipp::Communicator::custom(1, 3, [&](float* d, std::size_t n) {
    ++calls;
    for (std::size_t i = 0; i < n; ++i) d[i] *= 2;
  });
  float x[3] = {1, 2, 3};
  c.reduce_sum_to_root(x, 3);
  if (calls != 1 || x[2] != 6 || c.rank() != 1 || c.size() != 3) return 1;
  try {
    bipp::Communicator::custom(3, 3, nullptr);
    return 1;
  } catch (const bipp::InvalidParameterError&) {
  }
  return 0;
}
