// Autotuner and the table of tunable launch parameters (tune.hpp).
//
// The reference's only launch-shape logic is a fixed block-size ladder for its direct sum
// (src/gpu/kernels/nuft_sum.cu:73-84); here the shapes that matter for the batched
// pipeline are measured on the caller's own workload: the points per spreading work item
// and the spreader's resident CTAs per SM, the threads of the per-matrix
// tridiagonalisation, the persistent grid of the tensor-core virtual visibilities, and the
// input split of the direct sum. The tuner walks the parameters one at a time (coordinate
// descent), times each candidate with CUDA events around a full pipeline call on the
// caller's sample steps, keeps the fastest, and leaves the pipeline's images as they were
// before the call.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "bipp_b200.h"
#include "context.hpp"
#include "tune.hpp"

namespace bippb200 {
namespace {

struct Param {
  const char* name;
  int def;
  std::vector<int> candidates;
  const char* what;
  int value;
};

std::mutex g_tuneMu;
bool g_fileLoaded = false;

std::vector<Param>& table() {
  static std::vector<Param> t = {
      {"spread.items_cap", 2048, {2048, 4096, 8192}, "points per spreading work item (heavier tiles are split)", 0},
      {"spread.ctas_per_sm", 8, {2, 4, 8}, "resident tensor-core spreading CTAs per SM (at most 512 / TMEM columns)",
       0},
      {"spread.stages", 2, {1, 2},
       "operand stages of the tensor-core spreader (2: a phase is built while the previous one's MMAs run)", 0},
      {"spread.operands", 2, {0, 1, 2},
       "tensor-core spreader operands: 0 tf32 split, A in shared memory; 1 tf32 split, A in tensor memory "
       "(tcgen05.st by each thread); 2 FP16 hi/lo (kind::f16), values scaled per channel",
       0},
      {"spread.schedule", 1, {0, 1},
       "spreading work items: 0 round-robin over the persistent CTAs, 1 heaviest first from a work counter", 0},
      {"hetrd.threads", 0, {0, 256, 512, 1024}, "threads per matrix in the tridiagonalisation (0: by matrix size)", 0},
      {"hetrd.ctas_pct", 0, {0, 50, 75, 100, 150},
       "persistent tridiagonalisation CTAs in percent of the SM count (0: one CTA per matrix)", 0},
      {"tridiag.threads", 0, {0, 128, 256},
       "threads per matrix of the tridiagonal eigenpairs (0: 128 for a range of eigenpairs, 256 for all)", 0},
      {"bt.columns", 16, {16, 32},
       "eigenvector columns per CTA of the blocked back-transform (32: 512 threads, up to 512 rows; "
       "not autotuned: 6 % faster back-transform but a slower whole call on the 2048-step batch)",
       0},
      {"vv.ctas_per_sm", 3, {1, 2, 3}, "persistent tensor-core virtual-visibility CTAs per SM", 0},
      {"direct.ctas_per_sm", 4, {2, 4, 8}, "direct-sum CTAs per SM below which the inputs are split", 0},
      {"nufft.fft", 1, {0, 1},
       "inverse FFT of the w-planes: 1 = pruned two-pass transform that computes only the cells the pixels read "
       "(when the grid sizes have a plan), 0 = full 2-D cuFFT transform (not autotuned)",
       0},
      {"nufft.grid_per_1024", 1792, {1680, 1728, 1792},
       "NUFFT fine-grid cells per 1024 pixels (oversampling x 1024; read when a NUFFT is set up; not autotuned, "
       "as it trades accuracy for speed)",
       0},
  };
  static bool init = false;
  if (!init) {
    for (auto& p : t) p.value = p.def;
    init = true;
  }
  return t;
}

Param* find(const char* name) {
  for (auto& p : table())
    if (std::strcmp(p.name, name) == 0) return &p;
  return nullptr;
}

void set_value(const char* name, int value) {
  Param* p = find(name);
  if (!p) throw Error(BIPP_INVALID_PARAMETER_ERROR, std::string("unknown tunable parameter: ") + name);
  if (std::find(p->candidates.begin(), p->candidates.end(), value) == p->candidates.end())
    throw Error(BIPP_INVALID_PARAMETER_ERROR, std::string("value not among the candidates of ") + name);
  p->value = value;
}

// "name value" lines; '#' starts a comment
void load_file(const char* path) {
  std::ifstream in(path);
  if (!in) throw Error(BIPP_INVALID_PARAMETER_ERROR, std::string("cannot read tuning file: ") + path);
  std::string line;
  while (std::getline(in, line)) {
    const auto hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    std::istringstream ls(line);
    std::string name;
    int value;
    if (!(ls >> name)) continue;
    if (!(ls >> value)) throw Error(BIPP_INVALID_PARAMETER_ERROR, "malformed tuning line: " + line);
    set_value(name.c_str(), value);
  }
}

void ensure_file_loaded() {
  if (g_fileLoaded) return;
  g_fileLoaded = true;
  if (const char* f = std::getenv("BIPP_B200_TUNING_FILE"))
    if (*f) load_file(f);
}

}  // namespace

int tuned(const char* name) {
  std::lock_guard<std::mutex> lk(g_tuneMu);
  ensure_file_loaded();
  Param* p = find(name);
  if (!p) throw Error(BIPP_INVALID_PARAMETER_ERROR, std::string("unknown tunable parameter: ") + name);
  return p->value;
}

void set_tuned(const char* name, int value) {
  std::lock_guard<std::mutex> lk(g_tuneMu);
  ensure_file_loaded();
  set_value(name, value);
}

std::vector<int> tuning_candidates(const char* name) {
  std::lock_guard<std::mutex> lk(g_tuneMu);
  Param* p = find(name);
  if (!p) throw Error(BIPP_INVALID_PARAMETER_ERROR, std::string("unknown tunable parameter: ") + name);
  return p->candidates;
}

}  // namespace bippb200

using namespace bippb200;

extern "C" {

BippError bipp_tuning_get(const char* name, int* value) {
  return guard([&] {
    require(name && value, "null pointer", BIPP_INVALID_POINTER_ERROR);
    *value = tuned(name);
  });
}

BippError bipp_tuning_set(const char* name, int value) {
  return guard([&] {
    require(name != nullptr, "null pointer", BIPP_INVALID_POINTER_ERROR);
    std::lock_guard<std::mutex> lk(g_tuneMu);
    ensure_file_loaded();
    set_value(name, value);
  });
}

BippError bipp_tuning_describe(char* out, size_t len) {
  return guard([&] {
    require(out != nullptr && len > 0, "null pointer", BIPP_INVALID_POINTER_ERROR);
    std::lock_guard<std::mutex> lk(g_tuneMu);
    ensure_file_loaded();
    std::ostringstream os;
    for (const auto& p : table()) {
      os << p.name << " " << p.value << " [";
      for (size_t i = 0; i < p.candidates.size(); ++i) os << (i ? " " : "") << p.candidates[i];
      os << "] " << p.what << "\n";
    }
    const std::string s = os.str();
    require(s.size() < len, "output buffer too small");
    std::memcpy(out, s.c_str(), s.size() + 1);
  });
}

BippError bipp_tuning_save(const char* path) {
  return guard([&] {
    require(path != nullptr, "null pointer", BIPP_INVALID_POINTER_ERROR);
    std::lock_guard<std::mutex> lk(g_tuneMu);
    ensure_file_loaded();
    std::ofstream out(path);
    require((bool)out, "cannot write the tuning file");
    out << "# bipp_b200 tuned launch parameters (name value)\n";
    for (const auto& p : table()) out << p.name << " " << p.value << "\n";
  });
}

BippError bipp_tuning_load(const char* path) {
  return guard([&] {
    require(path != nullptr, "null pointer", BIPP_INVALID_POINTER_ERROR);
    std::lock_guard<std::mutex> lk(g_tuneMu);
    g_fileLoaded = true;
    load_file(path);
  });
}

BippError bipp_tuning_reset(void) {
  return guard([&] {
    std::lock_guard<std::mutex> lk(g_tuneMu);
    g_fileLoaded = true;
    for (auto& p : table()) p.value = p.def;
  });
}

}  // extern "C"
