// bipp::image_synthesis of the C++ API under Communicator::world(): every rank images its
// block of the samples and rank 0 receives the sum (the reference splits and MPI_Reduces,
// src/image_synthesis.cpp:75-80, 140-163). An in-memory Dataset, ImageProp and ImageData
// over raw files written by the test; rank 0 writes the images ([tags][pixels] float) to
// <out>. usage: multirank_check <dir> <nSamples> <nAnt> <nBeam> <nPixel> <out>
#include <bipp/bipp.hpp>

#include <complex>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <string>
#include <vector>

template <typename T>
static std::vector<T> read(const std::string& path, std::size_t n) {
  std::vector<T> v(n);
  std::ifstream f(path, std::ios::binary);
  f.read(reinterpret_cast<char*>(v.data()), n * sizeof(T));
  if (!f) throw std::runtime_error("cannot read " + path);
  return v;
}

struct FileDataset : bipp::Dataset {
  std::size_t ns, na, nb;
  std::vector<std::complex<float>> v;
  std::vector<float> d, uvw_, wl_, scale_;
  std::string desc = "test dataset";
  FileDataset(const std::string& dir, std::size_t s, std::size_t a, std::size_t b)
      : ns(s), na(a), nb(b), v(read<std::complex<float>>(dir + "/v.bin", s * a * b)), d(read<float>(dir + "/d.bin", s * b)),
        uvw_(read<float>(dir + "/uvw.bin", s * a * a * 3)), wl_(read<float>(dir + "/wl.bin", s)),
        scale_(read<float>(dir + "/scale.bin", s)) {}
  const std::string& description() const override { return desc; }
  std::size_t num_samples() const override { return ns; }
  std::size_t num_antenna() const override { return na; }
  std::size_t num_beam() const override { return nb; }
  void eig_vec(std::size_t i, std::complex<float>* out, std::size_t ldv) override {
    for (std::size_t c = 0; c < nb; ++c)
      for (std::size_t r = 0; r < na; ++r) out[r + c * ldv] = v[i * na * nb + r + c * na];
  }
  void eig_val(std::size_t i, float* out) override {
    for (std::size_t c = 0; c < nb; ++c) out[c] = d[i * nb + c];
  }
  void uvw(std::size_t i, float* out, std::size_t ld) override {
    const std::size_t m = na * na;
    for (std::size_t c = 0; c < 3; ++c)
      for (std::size_t k = 0; k < m; ++k) out[k + c * ld] = uvw_[i * m * 3 + k + c * m];
  }
  float wl(std::size_t i) override { return wl_[i]; }
  float time_stamp(std::size_t i) override { return (float)i; }
  float scale(std::size_t i) override { return scale_[i]; }
  float ra_deg() const override { return 0.f; }
  float dec_deg() const override { return 0.f; }
};

struct FileImageProp : bipp::ImageProp {
  std::size_t np;
  std::vector<float> lmn;
  FileImageProp(const std::string& dir, std::size_t n) : np(n), lmn(read<float>(dir + "/lmn.bin", n * 3)) {}
  void pixel_lmn(float* out, std::size_t ld) override {
    for (std::size_t c = 0; c < 3; ++c)
      for (std::size_t p = 0; p < np; ++p) out[p + c * ld] = lmn[p + c * np];
  }
  std::unordered_map<std::string, MetaType> meta_data() const override { return {}; }
  void set_meta(const std::string&, const MetaType&) override {}
  std::size_t width() const override { return np; }
  std::size_t height() const override { return 1; }
  float fov_deg() const override { return 10.f; }
};

struct MemImageData : bipp::ImageData {
  std::size_t np;
  std::map<std::string, std::vector<float>> img;
  explicit MemImageData(std::size_t n) : np(n) {}
  std::vector<std::string> tags() const override {
    std::vector<std::string> t;
    for (auto& [k, v] : img) t.push_back(k);
    return t;
  }
  std::size_t num_tags() const override { return img.size(); }
  void get(const std::string& tag, float* out) override { std::copy(img[tag].begin(), img[tag].end(), out); }
  void set(const std::string& tag, const float* in) override { img[tag].assign(in, in + np); }
  std::size_t width() const override { return np; }
  std::size_t height() const override { return 1; }
  float fov_deg() const override { return 10.f; }
  float ra_deg() const override { return 0.f; }
  float dec_deg() const override { return 0.f; }
};

int main(int argc, char** argv) {
  if (argc < 7) return 2;
  const std::string dir = argv[1], out = argv[6];
  const std::size_t ns = std::strtoull(argv[2], nullptr, 10), na = std::strtoull(argv[3], nullptr, 10),
                    nb = std::strtoull(argv[4], nullptr, 10), np = std::strtoull(argv[5], nullptr, 10);
  try {
    FileDataset ds(dir, ns, na, nb);
    FileImageProp prop(dir, np);
    MemImageData images(np);
    const auto ev = read<float>(dir + "/ev.bin", 2 * ns * nb);   // [tag][sample][beam]
    bipp::Selection sel;
    const char* tags[2] = {"lvl0", "lvl1"};
    // samples listed in reverse order: the library sorts them by id
    for (int t = 0; t < 2; ++t)
      for (std::size_t i = ns; i-- > 0;) sel[tags[t]].emplace_back(i, ev.data() + (t * ns + i) * nb);
    bipp::Context ctx(BIPP_PU_GPU, bipp::Communicator::world());
    bipp::NufftSynthesisOptions opt;
    opt.set_tolerance(1e-6f);
    opt.set_normalize_image(true);
    bipp::image_synthesis(ctx, opt, ds, sel, prop, images);
    if (ctx.communicator().rank() == 0) {
      std::ofstream f(out, std::ios::binary);
      for (int t = 0; t < 2; ++t) f.write(reinterpret_cast<const char*>(images.img.at(tags[t]).data()), np * 4);
    } else if (images.num_tags() != 0) {
      std::fprintf(stderr, "rank > 0 wrote images\n");
      return 1;
    }
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
