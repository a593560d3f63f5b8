// Calls the bipp C++ API of this library the way the reference's test does
// (tests/test_nufft_synthesis_lofar.cpp:152-156): eigh_gram<float/double> on raw inputs
// read from files, writes eigenvalues and eigenvectors back as raw binary.
// usage: api_check <dir> <nAntenna> <nBeam> <wl>
#include <bipp/bipp.hpp>

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

template <typename T>
static std::vector<T> read(const std::string& path, std::size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(T));
  return v;
}

template <typename T>
static void write(const std::string& path, const std::vector<T>& v) {
  std::ofstream f(path, std::ios::binary);
  f.write(reinterpret_cast<const char*>(v.data()), v.size() * sizeof(T));
}

template <typename T>
static int run(const std::string& dir, std::size_t nA, std::size_t nB, T wl, const char* tag) {
  auto s = read<std::complex<double>>(dir + "/s.bin", nB * nB);
  auto w = read<std::complex<double>>(dir + "/w.bin", nA * nB);
  auto xyz = read<double>(dir + "/xyz.bin", nA * 3);
  std::vector<std::complex<T>> sT(s.begin(), s.end()), wT(w.begin(), w.end());
  std::vector<T> xT(xyz.begin(), xyz.end()), d(nB);
  std::vector<std::complex<T>> v(nA * nB);
  auto r = bipp::eigh_gram<T>(wl, nA, nB, sT.data(), nB, wT.data(), nA, xT.data(), nA, d.data(), v.data(), nA);
  write(dir + "/d_" + tag + ".bin", d);
  write(dir + "/v_" + tag + ".bin", v);
  std::vector<double> meta = {double(r.first), double(r.second)};
  write(dir + "/meta_" + tag + ".bin", meta);
  return 0;
}

int main(int argc, char** argv) {
  if (argc < 5) return 2;
  const std::string dir = argv[1];
  const std::size_t nA = std::strtoull(argv[2], nullptr, 10), nB = std::strtoull(argv[3], nullptr, 10);
  const double wl = std::strtod(argv[4], nullptr);
  try {
    bipp::Context ctx(BIPP_PU_AUTO);
    if (ctx.processing_unit() != BIPP_PU_GPU) return 3;
    run<float>(dir, nA, nB, (float)wl, "f32");
    run<double>(dir, nA, nB, wl, "f64");
    // error path: a CPU context is rejected with the reference's exception type
    try {
      bipp::Context cpu(BIPP_PU_CPU);
      return 4;
    } catch (const bipp::InvalidParameterError& e) {
      if (e.error_code() != BIPP_INVALID_PARAMETER_ERROR) return 5;
    }
  } catch (const bipp::GenericError& e) {
    std::fprintf(stderr, "bipp error %d: %s\n", (int)e.error_code(), e.what());
    return 1;
  }
  return 0;
}
