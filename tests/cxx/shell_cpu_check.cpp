// Host-side checks of the bipp C++ API shell that need no GPU: the exception types and
// codes a reference caller catches, the CPU processing unit rejected, a GPU context
// without a device, and Communicator::world() from the launcher's variables. Exits 0
// when every check holds, else prints the failed check and exits 1.
#include <bipp/bipp.hpp>

#include <cstdio>
#include <cstdlib>
#include <string>

static int failures = 0;

static void expect(bool ok, const char* what) {
  if (!ok) {
    std::fprintf(stderr, "FAILED: %s\n", what);
    ++failures;
  }
}

int main(int argc, char** argv) {
  const bool noGpu = argc > 1 && std::string(argv[1]) == "no-gpu";
  try {
    bipp::Context ctx(BIPP_PU_CPU);
    expect(false, "a CPU context is rejected");
  } catch (const bipp::InvalidParameterError& e) {
    expect(e.error_code() == BIPP_INVALID_PARAMETER_ERROR, "InvalidParameterError code");
    expect(std::string(e.what()).find("CPU") != std::string::npos, "message names the CPU");
  }
  if (noGpu) {
    try {
      bipp::Context ctx(BIPP_PU_GPU);
      expect(false, "a GPU context without a device fails");
    } catch (const bipp::GPUError& e) {  // GPUSupportError derives from GPUError
      expect(e.error_code() == BIPP_GPU_SUPPORT_ERROR, "GPUSupportError code");
    }
  }
  try {
    throw bipp::EigensolverError();
  } catch (const bipp::GenericError& e) {
    expect(e.error_code() == BIPP_EIGENSOLVER_ERROR, "EigensolverError caught as GenericError");
  }
  try {
    throw bipp::MPIError();
  } catch (const bipp::GPUError& e) {
    expect(e.error_code() == BIPP_MPI_ERROR, "MPIError caught as GPUError");
  }
  setenv("RANK", "2", 1);
  setenv("WORLD_SIZE", "4", 1);
  const auto w = bipp::Communicator::world();
  expect(w.rank() == 2 && w.size() == 4, "Communicator::world from RANK and WORLD_SIZE");
  const auto l = bipp::Communicator::local();
  expect(l.rank() == 0 && l.size() == 1, "Communicator::local");
  return failures ? 1 : 0;
}
