// NUFFT engine (lattice type-1 in l/m + type-3 in n), the collect/get plan of the
// reference's NUFFTInterface, the direct nuft_sum and the domain partition.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdlib>
#include <limits>
#include <numeric>
#include <string>
#include <vector>

#include "context.hpp"
#include "nufft.hpp"
#include "tune.hpp"

#include <cub/device/device_radix_sort.cuh>
#include "spread_tc.cuh"

namespace bippb200 {

#define B2_CUFFT(call)                                                                         \
  do {                                                                                         \
    cufftResult r_ = (call);                                                                   \
    if (r_ != CUFFT_SUCCESS) throw Error(BIPP_GPU_ERROR, std::string(#call) + " failed: " +    \
                                                             std::to_string((int)r_));        \
  } while (0)

// ---------------------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------------------
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.resize(n);
  w.resize(n);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p0 = 1, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      const double dp = n * (z * p1 - p0) / (z * z - 1);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    double p0 = 1, p1 = z;
    for (int k = 2; k <= n; ++k) {
      const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    const double dp = n * (z * p1 - p0) / (z * z - 1);
    x[i] = z;
    w[i] = 2.0 / ((1 - z * z) * dp * dp);
  }
}

// Exponential-of-semicircle kernel parameters for tolerance eps at oversampling sigma
// (the published FINUFFT rules): sigma = 2: W = ceil(log10(1/eps)) + 1, beta/W = 2.30
// (2.20, 2.26, 2.38 for W = 2, 3, 4); otherwise W = ceil(ln(1/eps) / (pi sqrt(1 - 1/sigma)))
// and beta/W = 0.97 pi (1 - 1/(2 sigma)).
void es_params(double eps, double sigma, int& W, float& beta) {
  const double e = std::max(eps, 1e-15);
  double bw;
  if (sigma == 2.0) {
    W = (int)std::ceil(std::log10(1.0 / e)) + 1;
    bw = 2.30;
    if (W == 2) bw = 2.20;
    else if (W == 3) bw = 2.26;
    else if (W == 4) bw = 2.38;
  } else {
    W = (int)std::ceil(std::log(1.0 / e) / (M_PI * std::sqrt(1.0 - 1.0 / sigma)));
    bw = 0.97 * M_PI * (1.0 - 0.5 / sigma);
  }
  W = std::max(2, std::min(W, kMaxW));
  beta = (float)(bw * W);
}

static int next_smooth(int n) {
  // smallest m >= n, m % 16 == 0, m = 2^a 3^b 5^c 7^d
  for (int m = std::max(16, n);; ++m) {
    if (m % 16) continue;
    int r = m;
    for (int p : {2, 3, 5, 7})
      while (r % p == 0) r /= p;
    if (r == 1) return m;
  }
}

Lattice fit_lattice(const std::vector<double>& l, const std::vector<double>& m) {
  Lattice L;
  const size_t P = l.size();
  if (P < 4) return L;
  // candidate Nb: first index where the b-direction step changes, else try sqrt(P) and divisors
  std::vector<int> cands;
  const int sq = (int)std::llround(std::sqrt((double)P));
  if ((size_t)sq * sq == P) cands.push_back(sq);
  for (int nb = 2; nb <= (int)P / 2 && cands.size() < 64; ++nb)
    if (P % nb == 0 && nb != sq) cands.push_back(nb);
  for (int nb : cands) {
    const int na = (int)(P / nb);
    if (na < 2) continue;
    const double Bl = (l[nb - 1] - l[0]) / (nb - 1), Bm = (m[nb - 1] - m[0]) / (nb - 1);
    const double Al = (l[(size_t)(na - 1) * nb] - l[0]) / (na - 1), Am = (m[(size_t)(na - 1) * nb] - m[0]) / (na - 1);
    const double step = std::max(std::hypot(Bl, Bm), std::hypot(Al, Am));
    if (!(step > 0)) continue;
    double rl = 0, rm = 0;
    bool ok = true;
    for (int a = 0; a < na && ok; ++a)
      for (int b = 0; b < nb; ++b) {
        const size_t p = (size_t)a * nb + b;
        const double el = std::fabs(l[p] - (l[0] + a * Al + b * Bl));
        const double em = std::fabs(m[p] - (m[0] + a * Am + b * Bm));
        rl = std::max(rl, el);
        rm = std::max(rm, em);
        if (el > 1e-3 * step || em > 1e-3 * step) { ok = false; break; }
      }
    if (!ok) continue;
    // non-degenerate lattice
    const double det = Al * Bm - Am * Bl;
    if (std::fabs(det) < 1e-12 * step * step) continue;
    L.ok = true;
    L.Na = na; L.Nb = nb;
    L.l0 = l[0]; L.m0 = m[0]; L.Al = Al; L.Bl = Bl; L.Am = Am; L.Bm = Bm;
    L.maxResidL = rl; L.maxResidM = rm;
    return L;
  }
  return L;
}

// ---------------------------------------------------------------------------------------
// NufftCore
// ---------------------------------------------------------------------------------------
NufftCore::~NufftCore() {
  for (auto& kv : plans_) cufftDestroy(kv.second);
}

// Plan of one pass of the pruned FFT over lines of n values keeping nout outputs, with its
// compiled kernel (false when n has none: the caller uses cuFFT). Radices: the odd factor
// first, then the power of two 2^a (a >= 4, as the grid sizes are multiples of 16) as 16s
// with a remainder of 8 x 4 (a = 5 left), 8, 4 or 2; a lone radix-16 stage becomes 4 x 4,
// so the first stage's reads precede a barrier that the last stage's in-place writes
// follow. Threads per line: the fewest warps with which no thread holds more than
// kFftMaxValues values in any stage. Lines per CTA: 256 threads for the row pass; 4 lines
// for the column pass (a warp reads 32-byte row segments).
static bool make_fft_plan(int n, int nout, bool columnPass, FftLinePlan& pl, FftLinesKernel& kernel) {
  kernel = nullptr;
  pl = FftLinePlan{};
  pl.n = n;
  pl.nout = nout;
  std::vector<int> r;
  int m = n;
  for (int f : {7, 5, 3})
    while (m % f == 0) {
      r.push_back(f);
      m /= f;
    }
  int a = 0;
  while (m % 2 == 0) {
    ++a;
    m /= 2;
  }
  if (m != 1 || a < 4 || nout < 1 || nout > n) return false;
  while (a >= 4 && a != 5) {
    r.push_back(16);
    a -= 4;
  }
  if (a == 5) {
    r.push_back(8);
    r.push_back(4);
  } else if (a == 3) {
    r.push_back(8);
  } else if (a == 2) {
    r.push_back(4);
  } else if (a == 1) {
    r.push_back(2);
  }
  if (r.size() == 1 && r[0] == 16) r = {4, 4};
  if (r.size() < 2 || r.size() > (size_t)kFftMaxStages) return false;
  int T = 32;
  for (;; T += 32) {
    if (T > 512) return false;
    bool ok = true;
    for (int R : r) ok = ok && (n / R + T - 1) / T <= kFftMaxValues / R;
    if (ok) break;
  }
  pl.ns = (int)r.size();
  for (int s = 0; s < pl.ns; ++s) pl.radix[s] = r[s];
  pl.threads = T;
  pl.lineStride = (fft_pad(n - 1) + 1 + 15) / 16 * 16 + 4;
  int G = columnPass ? std::min(4, 512 / T) : std::max(1, 256 / T);
  while (G > 1 && (size_t)G * pl.lineStride * sizeof(float2) > (size_t)227 * 1024) --G;
  if ((size_t)G * pl.lineStride * sizeof(float2) > (size_t)227 * 1024) return false;
  pl.lines = G;
  kernel = fft_lines_kernel_for(pl.radix, pl.ns, columnPass);
  return kernel != nullptr;
}

// batched inverse 2-D FFT of the (channel, plane) arrays of the slab
void NufftCore::inverse_fft(int slabPlanes, int planesUsed, float2* slab, bool pruned) {
  if (pruned) {
    FftLines L{};
    L.data = slab;
    L.planesUsed = planesUsed;
    L.slabPlanes = slabPlanes;
    L.planeStride = (long long)g_.nx * g_.ny;
    // pass 1: every row along x, keeping Nb outputs
    L.linesPerPlane = g_.ny;
    L.nLines = (long long)nch_ * planesUsed * g_.ny;
    L.lineStep = g_.nx;
    L.elemStep = 1;
    size_t smem = (size_t)rowPlan_.lines * rowPlan_.lineStride * sizeof(float2);
    count_launch();
    rowKernel_<<<(unsigned)((L.nLines + rowPlan_.lines - 1) / rowPlan_.lines),
                              rowPlan_.lines * rowPlan_.threads, smem, ctx_->stream>>>(rowPlan_, L,
                                                                                       fftTw_.get<float2>());
    B2_CHECK_LAUNCH();
    // pass 2: the Nb kept columns along y, keeping Na outputs
    L.linesPerPlane = g_.Nb;
    L.nLines = (long long)nch_ * planesUsed * g_.Nb;
    L.lineStep = 1;
    L.elemStep = g_.nx;
    smem = (size_t)colPlan_.lines * colPlan_.lineStride * sizeof(float2);
    count_launch();
    colKernel_<<<(unsigned)((L.nLines + colPlan_.lines - 1) / colPlan_.lines),
                             colPlan_.lines * colPlan_.threads, smem, ctx_->stream>>>(
        colPlan_, L, fftTw_.get<float2>() + g_.nx);
    B2_CHECK_LAUNCH();
    return;
  }
  const int batch = nch_ * slabPlanes;
  auto it = plans_.find(batch);
  if (it == plans_.end()) {
    cufftHandle h;
    int n[2] = {g_.ny, g_.nx};
    B2_CUFFT(cufftPlanMany(&h, 2, n, nullptr, 1, g_.nx * g_.ny, nullptr, 1, g_.nx * g_.ny, CUFFT_C2C, batch));
    B2_CUFFT(cufftSetStream(h, ctx_->stream));
    it = plans_.emplace(batch, h).first;
  }
  B2_CUFFT(cufftExecC2C(it->second, reinterpret_cast<cufftComplex*>(slab), reinterpret_cast<cufftComplex*>(slab),
                        CUFFT_INVERSE));
}

void NufftCore::setup(bipp_ctx_s* ctx, const Lattice& lat, const std::vector<double>& n, double eps, int nch,
                      const std::vector<double>* dl, const std::vector<double>* dm, double su, double sv,
                      int levels) {
  ctx_ = ctx;
  require(lat.ok, "pixel coordinates are not on a lattice");
  corrCapable_ = (dl != nullptr);
  require(nch >= 1 && nch * (corrCapable_ ? 3 : 1) <= kMaxChan, "too many NUFFT channels");
  nch_ = nch;
  levels_ = nch;
  (void)levels;
  eps_ = eps;
  g_ = NufftGeom{};
  g_.l0 = lat.l0; g_.m0 = lat.m0; g_.Al = lat.Al; g_.Bl = lat.Bl; g_.Am = lat.Am; g_.Bm = lat.Bm;
  g_.Na = lat.Na; g_.Nb = lat.Nb;
  // oversampling (tunable, fine cells per 1024 pixels along a lattice axis; the w axis
  // takes the same factor): 1792 / 1024 = 1.75 gives the same kernel width as 2 at the
  // tolerances of interest (W = 6 at 1e-5) on (7/8)^3 of the fine grid; 1728 and 1680 keep
  // W = 6 at 1e-5 on smaller grids, with less margin in the width rule
  const double sigma = tuned("nufft.grid_per_1024") / 1024.0;
  es_params(eps, sigma, g_.W, g_.beta);
  g_.nx = next_smooth((int)std::ceil(sigma * g_.Nb));
  g_.ny = next_smooth((int)std::ceil(sigma * g_.Na));
  g_.nx = std::max(g_.nx, 2 * g_.W);
  g_.ny = std::max(g_.ny, 2 * g_.W);
  g_.hx = 2.0 * M_PI / g_.nx;
  g_.hy = 2.0 * M_PI / g_.ny;
  fftPlansOk_ = make_fft_plan(g_.nx, g_.Nb, false, rowPlan_, rowKernel_) &&
                make_fft_plan(g_.ny, g_.Na, true, colPlan_, colKernel_);
  if (fftPlansOk_) {
    // the passes' shared memory, set once here rather than before every launch
    B2_CUDA(cudaFuncSetAttribute((const void*)rowKernel_, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((size_t)rowPlan_.lines * rowPlan_.lineStride * sizeof(float2))));
    B2_CUDA(cudaFuncSetAttribute((const void*)colKernel_, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)((size_t)colPlan_.lines * colPlan_.lineStride * sizeof(float2))));
    std::vector<float2> tw((size_t)g_.nx + g_.ny);
    for (int i = 0; i < g_.nx; ++i)
      tw[i] = make_float2((float)std::cos(2.0 * M_PI * i / g_.nx), (float)std::sin(2.0 * M_PI * i / g_.nx));
    for (int i = 0; i < g_.ny; ++i)
      tw[(size_t)g_.nx + i] =
          make_float2((float)std::cos(2.0 * M_PI * i / g_.ny), (float)std::sin(2.0 * M_PI * i / g_.ny));
    fftTw_.alloc(ctx, tw.size() * sizeof(float2));
    h2d(ctx, fftTw_.get(), tw.data(), tw.size() * sizeof(float2));
  }
  const long long P = (long long)g_.Na * g_.Nb;
  require((long long)n.size() == P, "pixel n size mismatch");
  double nmin = *std::min_element(n.begin(), n.end()), nmax = *std::max_element(n.begin(), n.end());
  g_.nc = 0.5 * (nmin + nmax);
  Sn_ = std::max(0.5 * (nmax - nmin), 1e-12);
  g_.hw = M_PI / (sigma * Sn_);
  g_.ihx = 1.0 / g_.hx;
  g_.ihy = 1.0 / g_.hy;
  g_.ihw = 1.0 / g_.hw;
  std::vector<double> nt(P);
  for (long long p = 0; p < P; ++p) nt[p] = n[p] - g_.nc;
  nTilde_.alloc(ctx, P * sizeof(double));
  h2d(ctx, nTilde_.get(), nt.data(), P * sizeof(double));
  corrTerms_ = false;
  su_ = su;
  sv_ = sv;
  if (corrCapable_) {
    dl_.alloc(ctx, P * sizeof(double));
    dm_.alloc(ctx, P * sizeof(double));
    h2d(ctx, dl_.get(), dl->data(), P * sizeof(double));
    h2d(ctx, dm_.get(), dm->data(), P * sizeof(double));
  }
  // deconvolution factors (independent of the points)
  std::vector<double> qx, qwt;
  gauss_legendre(2 * g_.W + 16, qx, qwt);
  qz_.alloc(ctx, qx.size() * sizeof(double));
  qw_.alloc(ctx, qwt.size() * sizeof(double));
  h2d(ctx, qz_.get(), qx.data(), qx.size() * sizeof(double));
  h2d(ctx, qw_.get(), qwt.data(), qwt.size() * sizeof(double));
  decon_.alloc(ctx, P * sizeof(double));
  count_launch();
  decon_kernel<<<std::min<long long>(4096, (P + 255) / 256), 256, 0, ctx->stream>>>(
      g_, nTilde_.get<double>(), qz_.get<double>(), qw_.get<double>(), (int)qx.size(), decon_.get<double>());
  B2_CHECK_LAUNCH();
  acc_.alloc(ctx, (size_t)levels_ * (corrCapable_ ? 3 : 1) * P * sizeof(float2));
  zeroAcc_.alloc(ctx, kMaxChan * sizeof(double));
  sync(ctx);
}

void NufftCore::set_corr(bool on, double su, double sv) {
  corrTerms_ = on && corrCapable_;
  nch_ = corrTerms_ ? 3 * levels_ : levels_;
  su_ = su > 0 ? su : 1.0;
  sv_ = sv > 0 ? sv : 1.0;
}

void NufftCore::begin(double wmin, double wmax) {
  g_.wc = 0.5 * (wmin + wmax);
  const double Xw = std::max(0.5 * (wmax - wmin), 0.0);
  g_.jc = (int)std::ceil(Xw / g_.hw + 0.5 * g_.W) + 1;
  int nw = 2 * g_.jc + 1;
  nw = ((nw + kTW - 1) / kTW) * kTW;
  g_.nw = nw;
  g_.ntx = g_.nx / kTX;
  g_.nty = g_.ny / kTY;
  g_.ntw = g_.nw / kTW;
  nkeys_ = (long long)g_.ntx * g_.nty * g_.ntw * 8;
  require(nkeys_ < (1ll << 31) - 2, "NUFFT grid too large");
  counts_.ensure(ctx_, (nkeys_ + 1) * sizeof(int));
  B2_CUDA(cudaMemsetAsync(counts_.get(), 0, (nkeys_ + 1) * sizeof(int), ctx_->stream));
  B2_CUDA(cudaMemsetAsync(zeroAcc_.get(), 0, kMaxChan * sizeof(double), ctx_->stream));
}

void NufftCore::end_count(long long nPoints) {
  require(nPoints < (1ll << 31) - 1, "too many NUFFT points in one transform");
  const long long n = nkeys_;
  offsets_.ensure(ctx_, (n + 1) * sizeof(int));
  cursor_.ensure(ctx_, (n + 1) * sizeof(int));
  const long long per = (long long)kScanThreads * kScanItems;
  const int nb = (int)((n + per - 1) / per);
  blockSums_.ensure(ctx_, (nb + 1) * sizeof(int));
  count_launch();
  scan_partial_kernel<<<nb, kScanThreads, 0, ctx_->stream>>>(counts_.get<int>(), offsets_.get<int>(), n,
                                                             blockSums_.get<int>());
  count_launch();
  scan_blocksums_kernel<<<1, 1024, 0, ctx_->stream>>>(blockSums_.get<int>(), nb, offsets_.get<int>() + n);
  count_launch();
  scan_add_kernel<<<nb, 1024, 0, ctx_->stream>>>(offsets_.get<int>(), n, blockSums_.get<int>(), cursor_.get<int>());
  B2_CHECK_LAUNCH();
  valStride_ = std::max<long long>(nPoints, 1);
  rec_.ensure(ctx_, valStride_ * sizeof(PtRec));
  vals_.ensure(ctx_, (size_t)nch_ * valStride_ * sizeof(float2));
}

template <int CH, int W>
static void launch_spread_w(const NufftGeom& g, int nItems, size_t smem, cudaStream_t st, const int* offs,
                            const PtRec* rec, const float2* vals, long long vs, int nch, const SpreadItem* items,
                            int tw0, int slabPlanes, float2* out) {
  auto k = spread_warp_kernel<CH, W>;
  smem_optin(k, smem);
  count_launch();
  k<<<nItems, kSpreadThreads, smem, st>>>(g, offs, rec, vals, vs, nch, items, tw0, slabPlanes, out);
}

template <int CH>
static void launch_spread(const NufftGeom& g, int nItems, size_t smem, cudaStream_t st, const int* offs,
                          const PtRec* rec, const float2* vals, long long vs, int nch, const SpreadItem* items, int tw0,
                          int slabPlanes, float2* out) {
  switch (g.W) {
#define B2_W(w) \
  case w: launch_spread_w<CH, w>(g, nItems, smem, st, offs, rec, vals, vs, nch, items, tw0, slabPlanes, out); break;
    B2_W(2) B2_W(3) B2_W(4) B2_W(5) B2_W(6) B2_W(7) B2_W(8) B2_W(9)
#undef B2_W
    default: throw Error(BIPP_INTERNAL_ERROR, "unsupported NUFFT kernel width");
  }
}

// tensor-core spreading (4 or 8 channels): persistent CTAs, as many per SM as tensor
// memory allows
template <int CH, int STAGES, bool AT, bool F16>
static void launch_spread_tc(const NufftGeom& g, int nItems, cudaStream_t st, const int* offs, const PtRec* rec,
                             const float2* vals, long long vs, int nch, const SpreadItem* items, int tw0,
                             int slabPlanes, float2* out, int* errFlag, int* workCounter, const unsigned* valScale) {
  using S = TcShape<CH, STAGES, AT, F16>;
  int dev = 0, sms = 148;
  B2_CUDA(cudaGetDevice(&dev));
  B2_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  smem_optin(spread_tc_kernel<CH, STAGES, AT, F16>, S::Smem);
  // never more CTAs per SM than tensor memory holds (a CTA beyond that would wait in its
  // allocation until another one exits)
  const int grid = std::max(1, std::min(nItems, sms * std::min(S::MinBlocks, tuned("spread.ctas_per_sm"))));
  count_launch();
  spread_tc_kernel<CH, STAGES, AT, F16><<<grid, kTcThreads, S::Smem, st>>>(
      g, offs, rec, vals, vs, nch, items, nItems, tw0, slabPlanes, out, errFlag, workCounter, valScale);
}

// BIPP_B200_SPREAD=warp selects the shared-memory-atomic spreader for every channel count
static bool use_tensor_core_spread(int nch) {
  const char* e = std::getenv("BIPP_B200_SPREAD");
  if (e && std::string(e) == "warp") return false;
  return nch <= kTcMaxChan;
}


// exclusive scan of n ints on the stream; out[n] = total
void NufftCore::exclusive_scan(const int* in, int* out, long long n) {
  const long long per = (long long)kScanThreads * kScanItems;
  const int nb = (int)((n + per - 1) / per);
  itemSums_.ensure(ctx_, (nb + 1) * sizeof(int));
  count_launch();
  scan_partial_kernel<<<nb, kScanThreads, 0, ctx_->stream>>>(in, out, n, itemSums_.get<int>());
  count_launch();
  scan_blocksums_kernel<<<1, 1024, 0, ctx_->stream>>>(itemSums_.get<int>(), nb, out + n);
  count_launch();
  scan_add_kernel<<<nb, 1024, 0, ctx_->stream>>>(out, n, itemSums_.get<int>(), nullptr);
  B2_CHECK_LAUNCH();
}

void NufftCore::execute(float* image, long long ldImage, double* stageMs) {
  const long long P = num_pixels();
  const size_t planeBytes = (size_t)g_.nx * g_.ny * sizeof(float2);
  // slab size under a memory budget
  size_t freeB = 0, totalB = 0;
  B2_CUDA(cudaMemGetInfo(&freeB, &totalB));
  // grid slab budget: a quarter of free memory, at most 8 GB (BIPP_B200_SLAB_BYTES lowers it)
  size_t cap = (size_t)8 << 30;
  if (const char* e = std::getenv("BIPP_B200_SLAB_BYTES")) cap = std::max<size_t>(1, std::strtoull(e, nullptr, 10));
  const size_t budget = std::min<size_t>(std::max<size_t>(freeB / 4, planeBytes * kTW * nch_), cap);
  int slabTiles = (int)std::max<size_t>(1, budget / (planeBytes * kTW * nch_));
  slabTiles = std::min(slabTiles, g_.ntw);
  const int nslab = (g_.ntw + slabTiles - 1) / slabTiles;
  slabTiles = (g_.ntw + nslab - 1) / nslab;
  slabTiles_ = slabTiles;
  const int slabPlanes = slabTiles * kTW;
  grid_.ensure(ctx_, (size_t)nch_ * slabPlanes * planeBytes);
  B2_CUDA(cudaMemsetAsync(acc_.get(), 0, (size_t)nch_ * P * sizeof(float2), ctx_->stream));
  // per-tile loads -> work items (non-empty tiles, heavy tiles split in parts), built on
  // the device: parts per tile, exclusive scan -> item offsets, fill; tiles are numbered
  // slab by slab, so a slab's items are one contiguous range
  const int ntiles = g_.ntx * g_.nty * g_.ntw;
  load_.ensure(ctx_, (size_t)ntiles * sizeof(int));
  parts_.ensure(ctx_, (size_t)ntiles * sizeof(int));
  itemOff_.ensure(ctx_, (size_t)(ntiles + 1) * sizeof(int));
  // the tensor-core spreader writes every tile it spreads in one part; the other tiles of a
  // slab (empty, or split into parts that accumulate with atomics) are cleared first from
  // a compact list; the warp spreader works on a cleared slab
  const bool tc = use_tensor_core_spread(nch_);
  const bool prunedFft = fftPlansOk_ && tuned("nufft.fft") == 1;
  const int tb = std::min(8192, (ntiles + 255) / 256);
  clearFlag_.ensure(ctx_, (size_t)ntiles * sizeof(int));
  clearOff_.ensure(ctx_, (size_t)(ntiles + 1) * sizeof(int));
  clearList_.ensure(ctx_, (size_t)std::max(1, ntiles) * sizeof(int));
  count_launch();
  tile_load_kernel<<<tb, 256, 0, ctx_->stream>>>(g_, offsets_.get<int>(), load_.get<int>());
  splitCount_.ensure(ctx_, sizeof(int));
  B2_CUDA(cudaMemsetAsync(splitCount_.get(), 0, sizeof(int), ctx_->stream));
  count_launch();
  // points per spreading work item (tunable): heavier tiles are split so that no CTA
  // serialises the dense core of the uv plane (short baselines)
  const int spreadCap = tuned("spread.items_cap");
  tile_parts_kernel<<<tb, 256, 0, ctx_->stream>>>(ntiles, load_.get<int>(), spreadCap, parts_.get<int>(),
                                                  clearFlag_.get<int>(), splitCount_.get<int>());
  B2_CHECK_LAUNCH();
  exclusive_scan(parts_.get<int>(), itemOff_.get<int>(), ntiles);
  if (tc) {
    exclusive_scan(clearFlag_.get<int>(), clearOff_.get<int>(), ntiles);
    count_launch();
    clear_list_kernel<<<tb, 256, 0, ctx_->stream>>>(ntiles, clearFlag_.get<int>(), clearOff_.get<int>(),
                                                    clearList_.get<int>());
    B2_CHECK_LAUNCH();
  }
  const int tilesPerPlaneSet = g_.ntx * g_.nty;
  std::vector<int> slabBegin(nslab + 1, 0), clearBegin(nslab + 1, 0);
  for (int sl = 0; sl <= nslab; ++sl) {
    const int t = std::min(ntiles, sl * slabTiles * tilesPerPlaneSet);
    d2h(ctx_, &slabBegin[sl], itemOff_.get<int>() + t, sizeof(int));
    if (tc) d2h(ctx_, &clearBegin[sl], clearOff_.get<int>() + t, sizeof(int));
  }
  sync(ctx_);
  const int nItemsAll = slabBegin[nslab];
  items_.ensure(ctx_, std::max<size_t>(1, (size_t)nItemsAll) * sizeof(SpreadItem));
  count_launch();
  item_fill_kernel<<<tb, 256, 0, ctx_->stream>>>(ntiles, load_.get<int>(), parts_.get<int>(), itemOff_.get<int>(),
                                                 items_.get<SpreadItem>());
  B2_CHECK_LAUNCH();
  // load-ordered dynamic schedule (tunable): the items of every slab sorted heaviest
  // first, handed out by a work counter per slab launch
  const bool dynamic = tc && tuned("spread.schedule") == 1 && nItemsAll > 0;
  if (dynamic) {
    const int tilesPerSlab = slabTiles * g_.ntx * g_.nty;
    itemKeys_.ensure(ctx_, 2 * (size_t)nItemsAll * sizeof(unsigned));
    itemsAlt_.ensure(ctx_, (size_t)nItemsAll * sizeof(SpreadItem));
    count_launch();
    item_key_kernel<<<std::min(8192, (nItemsAll + 255) / 256), 256, 0, ctx_->stream>>>(
        nItemsAll, items_.get<SpreadItem>(), tilesPerSlab, itemKeys_.get<unsigned>());
    B2_CHECK_LAUNCH();
    int endBit = 20;
    while ((1 << (endBit - 20)) <= nslab && endBit < 32) ++endBit;
    size_t tmpBytes = 0;
    B2_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tmpBytes, itemKeys_.get<unsigned>(),
                                            itemKeys_.get<unsigned>() + nItemsAll, items_.get<SpreadItem>(),
                                            itemsAlt_.get<SpreadItem>(), nItemsAll, 0, endBit, ctx_->stream));
    sortTmp_.ensure(ctx_, std::max<size_t>(tmpBytes, 16));
    B2_CUDA(cub::DeviceRadixSort::SortPairs(sortTmp_.get(), tmpBytes, itemKeys_.get<unsigned>(),
                                            itemKeys_.get<unsigned>() + nItemsAll, items_.get<SpreadItem>(),
                                            itemsAlt_.get<SpreadItem>(), nItemsAll, 0, endBit, ctx_->stream));
    B2_CUDA(cudaMemcpyAsync(items_.get(), itemsAlt_.get(), (size_t)nItemsAll * sizeof(SpreadItem),
                            cudaMemcpyDeviceToDevice, ctx_->stream));
    workCounters_.ensure(ctx_, (size_t)std::max(1, nslab) * sizeof(int));
    B2_CUDA(cudaMemsetAsync(workCounters_.get(), 0, (size_t)std::max(1, nslab) * sizeof(int), ctx_->stream));
  }
  {
    int total = 0, split = 0;
    d2h(ctx_, &total, offsets_.get<int>() + nkeys_, sizeof(int));
    d2h(ctx_, &split, splitCount_.get<int>(), sizeof(int));
    sync(ctx_);
    lastPoints = total;
    lastSplitTiles = split;
    lastSlabs = nslab;
    lastItems = nItemsAll;
    lastGridBytes = (long long)g_.ntw * kTW * (long long)planeBytes * nch_;
  }
  // spreader operands (tunable): 0 tf32 split with A in shared memory, 1 with A in tensor
  // memory, 2 FP16 hi/lo (values scaled per channel by their largest magnitude)
  const int operands = tc ? tuned("spread.operands") : 0;
  valScale_.ensure(ctx_, kMaxChan * sizeof(unsigned));
  if (operands == 2) {
    B2_CUDA(cudaMemsetAsync(valScale_.get(), 0, kMaxChan * sizeof(unsigned), ctx_->stream));
    if (lastPoints > 0) {
      count_launch();
      value_scale_kernel<<<std::min<long long>(4096, (lastPoints + 255) / 256), 256, 0, ctx_->stream>>>(
          offsets_.get<int>() + nkeys_, vals_.get<float2>(), nch_, valScale_.get<unsigned>());
      B2_CHECK_LAUNCH();
    }
  }
  const size_t smem = (size_t)nch_ * 2 * kTileCells * sizeof(float);
  errFlag_.ensure(ctx_, sizeof(int));
  B2_CUDA(cudaMemsetAsync(errFlag_.get(), 0, sizeof(int), ctx_->stream));
  cudaEvent_t ev[5];
  if (stageMs)
    for (auto& e : ev) B2_CUDA(cudaEventCreate(&e));
  float tSpread = 0, tFft = 0, tW = 0, tClear = 0;
  for (int sl = 0; sl < nslab; ++sl) {
    const int tw0 = sl * slabTiles;
    const int tiles = std::min(slabTiles, g_.ntw - tw0);
    const int nItems = slabBegin[sl + 1] - slabBegin[sl];
    if (stageMs) B2_CUDA(cudaEventRecord(ev[4], ctx_->stream));
    if (!tc) {
      B2_CUDA(cudaMemsetAsync(grid_.get(), 0, (size_t)nch_ * slabPlanes * planeBytes, ctx_->stream));
    } else if (clearBegin[sl + 1] > clearBegin[sl]) {
      count_launch();
      clear_tiles_kernel<<<clearBegin[sl + 1] - clearBegin[sl], kTcThreads, 0, ctx_->stream>>>(
          g_, clearList_.get<int>() + clearBegin[sl], tw0, slabPlanes, nch_, grid_.get<float2>());
      B2_CHECK_LAUNCH();
    }
    if (stageMs) B2_CUDA(cudaEventRecord(ev[0], ctx_->stream));
    if (nItems > 0 && tc) {
      const bool two = tuned("spread.stages") == 2;
      using L = decltype(&launch_spread_tc<4, 1, false, false>);
      // [channels 4 / 8][operands: tf32 split with A in shared memory / in tensor memory /
      // FP16 hi-lo][stages 1 / 2]
      static const L table[2][3][2] = {
          {{launch_spread_tc<4, 1, false, false>, launch_spread_tc<4, 2, false, false>},
           {launch_spread_tc<4, 1, true, false>, launch_spread_tc<4, 2, true, false>},
           {launch_spread_tc<4, 1, false, true>, launch_spread_tc<4, 2, false, true>}},
          {{launch_spread_tc<8, 1, false, false>, launch_spread_tc<8, 2, false, false>},
           {launch_spread_tc<8, 1, true, false>, launch_spread_tc<8, 2, true, false>},
           {launch_spread_tc<8, 1, false, true>, launch_spread_tc<8, 2, false, true>}}};
      const L launch = table[nch_ <= 4 ? 0 : 1][operands][two ? 1 : 0];
      launch(g_, nItems, ctx_->stream, offsets_.get<int>(), rec_.get<PtRec>(), vals_.get<float2>(), valStride_, nch_,
             items_.get<SpreadItem>() + slabBegin[sl], tw0, slabPlanes, grid_.get<float2>(), errFlag_.get<int>(),
             dynamic ? workCounters_.get<int>() + sl : nullptr, valScale_.get<unsigned>());
      B2_CHECK_LAUNCH();
    } else if (nItems > 0) {
      const SpreadItem* it = items_.get<SpreadItem>() + slabBegin[sl];
      if (nch_ <= 4)
        launch_spread<4>(g_, nItems, smem, ctx_->stream, offsets_.get<int>(), rec_.get<PtRec>(), vals_.get<float2>(),
                         valStride_, nch_, it, tw0, slabPlanes, grid_.get<float2>());
      else
        launch_spread<kMaxChan>(g_, nItems, smem, ctx_->stream, offsets_.get<int>(), rec_.get<PtRec>(),
                                vals_.get<float2>(), valStride_, nch_, it, tw0, slabPlanes, grid_.get<float2>());
      B2_CHECK_LAUNCH();
    }
    if (stageMs) B2_CUDA(cudaEventRecord(ev[1], ctx_->stream));
    inverse_fft(slabPlanes, tiles * kTW, grid_.get<float2>(), prunedFft);
    if (stageMs) B2_CUDA(cudaEventRecord(ev[2], ctx_->stream));
    const int blocks = (int)std::min<long long>((P + 255) / 256, 65535);
    count_launch();
    auto wk = nch_ <= 4 ? wsum_kernel<4> : wsum_kernel<kMaxChan>;
    wk<<<blocks, 256, 0, ctx_->stream>>>(g_, grid_.get<float2>(), nch_, slabPlanes, tw0 * kTW, tiles * kTW,
                                         nTilde_.get<double>(), acc_.get<float2>(), P, prunedFft ? 1 : 0);
    B2_CHECK_LAUNCH();
    if (stageMs) {
      B2_CUDA(cudaEventRecord(ev[3], ctx_->stream));
      B2_CUDA(cudaEventSynchronize(ev[3]));
      float a, b, c, z;
      cudaEventElapsedTime(&a, ev[0], ev[1]);
      cudaEventElapsedTime(&b, ev[1], ev[2]);
      cudaEventElapsedTime(&c, ev[2], ev[3]);
      cudaEventElapsedTime(&z, ev[4], ev[0]);
      tSpread += a; tFft += b; tW += c; tClear += z;
    }
  }
  const int blocks = (int)std::min<long long>((P + 255) / 256, 65535);
  count_launch();
  finalize_kernel<<<blocks, 256, 0, ctx_->stream>>>(P, levels_, acc_.get<float2>(), P, decon_.get<double>(),
                                                    nTilde_.get<double>(), g_.wc, corrTerms_ ? 1 : 0,
                                                    dl_.get<double>(), dm_.get<double>(), su_, sv_, image, ldImage,
                                                    zeroAcc_.get<double>());
  B2_CHECK_LAUNCH();
  if (tc) {
    int err = 0;
    d2h(ctx_, &err, errFlag_.get(), sizeof(int));
    sync(ctx_);
    if (err) throw Error(BIPP_GPU_ERROR, "tensor-core spreading: MMA completion wait timed out");
  }
  if (stageMs) {
    stageMs[0] += tSpread;
    stageMs[1] += tFft;
    stageMs[2] += tW;
    stageMs[3] += tClear;
    for (auto& e : ev) cudaEventDestroy(e);
  }
}

static __global__ void f2d_kernel(const float* __restrict__ in, long long n, double* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

// ---------------------------------------------------------------------------------------
// min/max reduction of the scaled w coordinate of baseline points
// ---------------------------------------------------------------------------------------
__global__ void minmax_kernel(const float* __restrict__ x, long long n, double scale, double* __restrict__ out) {
  __shared__ double rmin[32], rmax[32];
  double lo = 1e300, hi = -1e300;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = (double)x[i] * scale;
    lo = fmin(lo, v);
    hi = fmax(hi, v);
  }
  lo = block_min(lo, rmin, 1e300);
  hi = block_max(hi, rmax, -1e300);
  if (threadIdx.x == 0) {
    out[2 * blockIdx.x] = lo;
    out[2 * blockIdx.x + 1] = hi;
  }
}

}  // namespace bippb200

// ---------------------------------------------------------------------------------------
// collect / get plan
// ---------------------------------------------------------------------------------------
using namespace bippb200;

struct bipp_nufft_s {
  bipp_ctx_s* ctx = nullptr;
  bipp_nufft_options opt{};
  size_t nPixel = 0, nImages = 0, nBaselines = 0, batch = 0, count = 0;
  bool lattice = false;
  NufftCore core;
  DevBuf uvw;        // [3][batch * nBaselines] float (scaled)
  DevBuf values;     // [nImages][batch * nBaselines] float2
  DevBuf lmnDev;     // [3][nPixel] double (direct path)
  DevBuf images;     // [nImages][nPixel] float
  DevBuf imagesD;    // [nImages][nPixel] double (direct path accumulation)
  DevBuf mm;         // min/max scratch
  bool double_in = false;
  double residL = 0, residM = 0;
};

static void nufft_transform_lattice(bipp_nufft_s* p, long long n, long long ld);

static void nufft_transform(bipp_nufft_s* p) {
  if (!p->count) return;
  bipp_ctx_s* ctx = p->ctx;
  const long long n = (long long)p->count * p->nBaselines;
  const long long ld = (long long)p->batch * p->nBaselines;
  if (p->lattice) {
    nufft_transform_lattice(p, n, ld);
  } else {
    // direct evaluation for pixels that are not on a lattice: FP64 phase, FP64 trig
    const double* lx = p->lmnDev.get<double>();
    DevBuf u64(ctx, 3 * n * sizeof(double));
    DevBuf v64(ctx, n * sizeof(double2));
    for (int c = 0; c < 3; ++c) {
      count_launch();
      f2d_kernel<<<256, 256, 0, ctx->stream>>>(p->uvw.get<float>() + c * ld, n, u64.get<double>() + c * n);
    }
    B2_CHECK_LAUNCH();
    const double* ud = u64.get<double>();
    const dim3 blocks = direct_sum_grid((long long)p->nPixel, (long long)n, ctx->smCount, tuned("direct.ctas_per_sm"));
    for (size_t im = 0; im < p->nImages; ++im) {
      count_launch();
      f2d_kernel<<<256, 256, 0, ctx->stream>>>(reinterpret_cast<const float*>(p->values.get<float2>() + im * ld), 2 * n,
                                               v64.get<double>());
      count_launch();
      direct_sum_kernel<double, double2, double, 1><<<blocks, kDirectThreads, 0, ctx->stream>>>(
          1.0, n, v64.get<double2>(), n, ud, ud + n, ud + 2 * n, (long long)p->nPixel, lx, lx + p->nPixel,
          lx + 2 * p->nPixel, p->imagesD.get<double>() + im * p->nPixel, (long long)p->nPixel, 1, 1);
      B2_CHECK_LAUNCH();
    }
  }
  p->count = 0;
}

static void host_minmax(bipp_ctx_s* ctx, const float* x, long long n, DevBuf& scratch, double& lo, double& hi) {
  const int blocks = 256;
  scratch.ensure(ctx, 2 * blocks * sizeof(double));
  count_launch();
  minmax_kernel<<<blocks, 256, 0, ctx->stream>>>(x, n, 1.0, scratch.get<double>());
  B2_CHECK_LAUNCH();
  std::vector<double> mm(2 * blocks);
  d2h(ctx, mm.data(), scratch.get(), mm.size() * sizeof(double));
  sync(ctx);
  lo = 1e300;
  hi = -1e300;
  for (int i = 0; i < blocks; ++i) {
    lo = std::min(lo, mm[2 * i]);
    hi = std::max(hi, mm[2 * i + 1]);
  }
}

// transform of the collected samples (lattice path); the non-lattice path is handled by
// nufft_transform's direct branch
static void nufft_transform_lattice(bipp_nufft_s* p, long long n, long long ld) {
  bipp_ctx_s* ctx = p->ctx;
  double umin, umax, vmin, vmax, wmin, wmax;
  host_minmax(ctx, p->uvw.get<float>(), n, p->mm, umin, umax);
  host_minmax(ctx, p->uvw.get<float>() + ld, n, p->mm, vmin, vmax);
  host_minmax(ctx, p->uvw.get<float>() + 2 * ld, n, p->mm, wmin, wmax);
  p->core.begin(0.0, std::max(-wmin, wmax));  // points are folded to w >= 0
  const double su = std::max(std::fabs(umin), std::fabs(umax)), sv = std::max(std::fabs(vmin), std::fabs(vmax));
  // first-order correction for the FP32 rounding of the pixel coordinates when the
  // residual phase could exceed a tenth of the tolerance
  const double bound = p->residL * su + p->residM * sv;
  p->core.set_corr(bound > 0.1 * p->opt.tolerance, su, sv);
  const size_t groups = p->nImages;
  (void)groups;
  BaselinePoints bp{};
  bp.n = n;
  bp.uvw = p->uvw.get<float>();
  bp.lduvw = ld;
  bp.uvwScale = 1.0;
  bp.values = p->values.get<float2>();
  bp.ldv = ld;
  bp.levels = (int)p->nImages;
  const NufftGeom& g = p->core.geom();
  const int gb = (int)std::min<long long>((n + 255) / 256, 8192);
  count_launch();
  baseline_count_kernel<<<gb, 256, 0, ctx->stream>>>(g, bp, p->core.counts());
  B2_CHECK_LAUNCH();
  p->core.end_count(n);
  count_launch();
  baseline_scatter_kernel<<<gb, 256, 0, ctx->stream>>>(g, bp, p->core.cursor(), p->core.records(), p->core.values(),
                                                       p->core.value_stride(), p->core.sincos64() ? 1 : 0,
                                                       p->core.corr_terms() ? 1 : 0, p->core.su(), p->core.sv(),
                                                       p->core.zero_acc(), p->core.channels());
  B2_CHECK_LAUNCH();
  p->core.execute(p->images.get<float>(), (long long)p->nPixel);
}

__global__ void add_double_to_float_kernel(const double* __restrict__ a, long long n, float* __restrict__ b) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    b[i] += (float)a[i];
}

__global__ void d2f_kernel(const double* __restrict__ in, long long n, float* __restrict__ out) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}

namespace bippb200 {
float* nufft_stage_uvw(bipp_nufft_t p) { return p->uvw.get<float>() + p->count * p->nBaselines; }
float2* nufft_stage_values(bipp_nufft_t p, size_t im) {
  return p->values.get<float2>() + im * (long long)p->batch * p->nBaselines + p->count * p->nBaselines;
}
long long nufft_stage_ld(bipp_nufft_t p) { return (long long)p->batch * p->nBaselines; }
void nufft_commit(bipp_nufft_t p) {
  ++p->count;
  if (p->count >= p->batch) nufft_transform(p);
}
}  // namespace bippb200

extern "C" {

BippError bipp_nufft_create(bipp_ctx_t ctx, const bipp_nufft_options* opt, size_t nPixel, const float* lmn,
                            size_t ldlmn, size_t nImages, size_t nBaselines, bipp_nufft_t* plan) {
  return guard([&] {
    require(ctx && opt && lmn && plan, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(nPixel > 0 && nImages > 0 && nBaselines > 0, "empty NUFFT");
    require(ldlmn >= nPixel, "invalid ldlmn");
    require(nImages <= 4, "at most 4 images per collector (create one collector per group of 4)");
    auto p = std::make_unique<bipp_nufft_s>();
    p->ctx = ctx;
    p->opt = *opt;
    p->nPixel = nPixel;
    p->nImages = nImages;
    p->nBaselines = nBaselines;
    size_t batch = opt->sampleBatchSize;
    if (batch == 0) batch = std::max<size_t>(1, (size_t)2000000000ull / (20 * nBaselines));
    p->batch = batch;
    std::vector<double> l(nPixel), m(nPixel), nn(nPixel);
    for (size_t i = 0; i < nPixel; ++i) {
      l[i] = lmn[i];
      m[i] = lmn[i + ldlmn];
      nn[i] = lmn[i + 2 * ldlmn];
    }
    Lattice lat = fit_lattice(l, m);
    p->lattice = lat.ok;
    if (lat.ok) {
      std::vector<double> dl(nPixel), dm(nPixel);
      for (int a = 0; a < lat.Na; ++a)
        for (int b = 0; b < lat.Nb; ++b) {
          const size_t q = (size_t)a * lat.Nb + b;
          dl[q] = l[q] - (lat.l0 + a * lat.Al + b * lat.Bl);
          dm[q] = m[q] - (lat.m0 + a * lat.Am + b * lat.Bm);
        }
      p->residL = lat.maxResidL;
      p->residM = lat.maxResidM;
      p->core.setup(ctx, lat, nn, std::max<double>(opt->tolerance, 1e-12), (int)nImages, &dl, &dm);
    } else {
      std::vector<double> h(3 * nPixel);
      for (size_t i = 0; i < nPixel; ++i) {
        h[i] = l[i];
        h[i + nPixel] = m[i];
        h[i + 2 * nPixel] = nn[i];
      }
      p->lmnDev.alloc(ctx, h.size() * sizeof(double));
      h2d(ctx, p->lmnDev.get(), h.data(), h.size() * sizeof(double));
      p->imagesD.alloc(ctx, nImages * nPixel * sizeof(double));
      p->imagesD.zero();
    }
    p->uvw.alloc(ctx, 3 * batch * nBaselines * sizeof(float));
    p->values.alloc(ctx, nImages * batch * nBaselines * sizeof(float2));
    p->images.alloc(ctx, nImages * nPixel * sizeof(float));
    p->images.zero();
    sync(ctx);
    ctx_retain(ctx);
    *plan = p.release();
  });
}

static void nufft_add(bipp_nufft_t plan, const void* uvw, size_t lduvw, const void* values, size_t ldvalues,
                      bool dbl) {
  require(plan && uvw && values, "null pointer", BIPP_INVALID_POINTER_ERROR);
  bipp_nufft_s* p = plan;
  require(lduvw >= p->nBaselines && ldvalues >= p->nBaselines, "invalid leading dimension");
  bipp_ctx_s* ctx = p->ctx;
  const size_t nB = p->nBaselines;
  const long long ld = (long long)p->batch * nB;
  const size_t off = p->count * nB;
  if (!dbl) {
    const float* u = static_cast<const float*>(uvw);
    for (int c = 0; c < 3; ++c) h2d(ctx, p->uvw.get<float>() + c * ld + off, u + c * lduvw, nB * sizeof(float));
    const std::complex<float>* v = static_cast<const std::complex<float>*>(values);
    for (size_t im = 0; im < p->nImages; ++im)
      h2d(ctx, p->values.get<float2>() + im * ld + off, v + im * ldvalues, nB * sizeof(float2));
  } else {
    // double input is rounded to the FP32 collection buffers
    const double* u = static_cast<const double*>(uvw);
    std::vector<float> tmp(nB);
    for (int c = 0; c < 3; ++c) {
      for (size_t i = 0; i < nB; ++i) tmp[i] = (float)u[i + c * lduvw];
      h2d(ctx, p->uvw.get<float>() + c * ld + off, tmp.data(), nB * sizeof(float));
      sync(ctx);
    }
    const std::complex<double>* v = static_cast<const std::complex<double>*>(values);
    std::vector<std::complex<float>> vt(nB);
    for (size_t im = 0; im < p->nImages; ++im) {
      for (size_t i = 0; i < nB; ++i) vt[i] = std::complex<float>((float)v[i + im * ldvalues].real(), (float)v[i + im * ldvalues].imag());
      h2d(ctx, p->values.get<float2>() + im * ld + off, vt.data(), nB * sizeof(float2));
      sync(ctx);
    }
  }
  sync(ctx);
  ++p->count;
  if (p->count >= p->batch) nufft_transform(p);
}


BippError bipp_nufft_add_s(bipp_nufft_t plan, const float* uvw, size_t lduvw, const void* values, size_t ldvalues) {
  return guard([&] { nufft_add(plan, uvw, lduvw, values, ldvalues, false); });
}
BippError bipp_nufft_add_d(bipp_nufft_t plan, const double* uvw, size_t lduvw, const void* values, size_t ldvalues) {
  return guard([&] { nufft_add(plan, uvw, lduvw, values, ldvalues, true); });
}

BippError bipp_nufft_get_image(bipp_nufft_t plan, size_t imgIdx, float* image) {
  return guard([&] {
    require(plan && image, "null pointer", BIPP_INVALID_POINTER_ERROR);
    bipp_nufft_s* p = plan;
    require(imgIdx < p->nImages, "image index out of range");
    nufft_transform(p);
    bipp_ctx_s* ctx = p->ctx;
    if (!p->lattice) {
      // fold the FP64 direct-sum accumulator into the float images
      count_launch();
      add_double_to_float_kernel<<<256, 256, 0, ctx->stream>>>(p->imagesD.get<double>(), (long long)(p->nImages * p->nPixel),
                                                              p->images.get<float>());
      B2_CHECK_LAUNCH();
      p->imagesD.zero();
    }
    d2h(ctx, image, p->images.get<float>() + imgIdx * p->nPixel, p->nPixel * sizeof(float));
    sync(ctx);
  });
}

BippError bipp_nufft_destroy(bipp_nufft_t plan) {
  return guard([&] {
    if (!plan) return;
    bipp_ctx_s* ctx = plan->ctx;
    delete plan;
    sync(ctx);
    ctx_release(ctx);
  });
}

BippError bipp_nuft_sum_s(bipp_ctx_t ctx, float alpha, size_t nIn, const void* input, const float* u, const float* v,
                          const float* w, size_t nOut, const float* x, const float* y, const float* z, float* out) {
  return guard([&] {
    require(ctx && input && u && v && w && x && y && z && out, "null pointer", BIPP_INVALID_POINTER_ERROR);
    if (!nOut) return;
    DevBuf dIn(ctx, nIn * sizeof(float2) + 16), dU(ctx, 3 * nIn * sizeof(float) + 16), dX(ctx, 3 * nOut * sizeof(float)),
        dO(ctx, nOut * sizeof(float));
    h2d(ctx, dIn.get(), input, nIn * sizeof(float2));
    h2d(ctx, dU.get<float>(), u, nIn * sizeof(float));
    h2d(ctx, dU.get<float>() + nIn, v, nIn * sizeof(float));
    h2d(ctx, dU.get<float>() + 2 * nIn, w, nIn * sizeof(float));
    h2d(ctx, dX.get<float>(), x, nOut * sizeof(float));
    h2d(ctx, dX.get<float>() + nOut, y, nOut * sizeof(float));
    h2d(ctx, dX.get<float>() + 2 * nOut, z, nOut * sizeof(float));
    h2d(ctx, dO.get(), out, nOut * sizeof(float));
    const dim3 blocks = direct_sum_grid((long long)nOut, (long long)nIn, ctx->smCount, tuned("direct.ctas_per_sm"));
    count_launch();
    direct_sum_kernel<float, float2, float, 1><<<blocks, kDirectThreads, 0, ctx->stream>>>(
        (double)alpha, (long long)nIn, dIn.get<float2>(), (long long)nIn, dU.get<float>(), dU.get<float>() + nIn,
        dU.get<float>() + 2 * nIn, (long long)nOut, dX.get<float>(), dX.get<float>() + nOut, dX.get<float>() + 2 * nOut,
        dO.get<float>(), (long long)nOut, 1, 0);
    B2_CHECK_LAUNCH();
    d2h(ctx, out, dO.get(), nOut * sizeof(float));
    sync(ctx);
  });
}

BippError bipp_nuft_sum_d(bipp_ctx_t ctx, double alpha, size_t nIn, const void* input, const double* u, const double* v,
                          const double* w, size_t nOut, const double* x, const double* y, const double* z, double* out) {
  return guard([&] {
    require(ctx && input && u && v && w && x && y && z && out, "null pointer", BIPP_INVALID_POINTER_ERROR);
    if (!nOut) return;
    DevBuf dIn(ctx, nIn * sizeof(double2) + 16), dU(ctx, 3 * nIn * sizeof(double) + 16),
        dX(ctx, 3 * nOut * sizeof(double)), dO(ctx, nOut * sizeof(double));
    h2d(ctx, dIn.get(), input, nIn * sizeof(double2));
    h2d(ctx, dU.get<double>(), u, nIn * sizeof(double));
    h2d(ctx, dU.get<double>() + nIn, v, nIn * sizeof(double));
    h2d(ctx, dU.get<double>() + 2 * nIn, w, nIn * sizeof(double));
    h2d(ctx, dX.get<double>(), x, nOut * sizeof(double));
    h2d(ctx, dX.get<double>() + nOut, y, nOut * sizeof(double));
    h2d(ctx, dX.get<double>() + 2 * nOut, z, nOut * sizeof(double));
    h2d(ctx, dO.get(), out, nOut * sizeof(double));
    const dim3 blocks = direct_sum_grid((long long)nOut, (long long)nIn, ctx->smCount, tuned("direct.ctas_per_sm"));
    count_launch();
    direct_sum_kernel<double, double2, double, 1><<<blocks, kDirectThreads, 0, ctx->stream>>>(
        alpha, (long long)nIn, dIn.get<double2>(), (long long)nIn, dU.get<double>(), dU.get<double>() + nIn,
        dU.get<double>() + 2 * nIn, (long long)nOut, dX.get<double>(), dX.get<double>() + nOut,
        dX.get<double>() + 2 * nOut, dO.get<double>(), (long long)nOut, 1, 1);
    B2_CHECK_LAUNCH();
    d2h(ctx, out, dO.get(), nOut * sizeof(double));
    sync(ctx);
  });
}

BippError bipp_nuft_sum_multi_device(bipp_ctx_t ctx, double alpha, size_t nIn, size_t nch, const void* values,
                                     size_t ldIn, const double* u, const double* v, const double* w, size_t nOut,
                                     const double* x, const double* y, const double* z, double* out, size_t ldOut,
                                     int fp64Trig) {
  return guard([&] {
    require(ctx && values && u && v && w && x && y && z && out, "null pointer", BIPP_INVALID_POINTER_ERROR);
    require(nch >= 1 && ldIn >= nIn && ldOut >= nOut, "invalid sizes");
    if (!nOut) return;
    const dim3 blocks = direct_sum_grid((long long)nOut, (long long)nIn, ctx->smCount, tuned("direct.ctas_per_sm"));
    for (size_t c0 = 0; c0 < nch; c0 += 4) {
      const int n = (int)std::min<size_t>(4, nch - c0);
      count_launch();
      direct_sum_kernel<double, float2, double, 4><<<blocks, kDirectThreads, 0, ctx->stream>>>(
          alpha, (long long)nIn, static_cast<const float2*>(values) + c0 * ldIn, (long long)ldIn, u, v, w,
          (long long)nOut, x, y, z, out + c0 * ldOut, (long long)ldOut, n, fp64Trig);
      B2_CHECK_LAUNCH();
    }
    sync(ctx);
  });
}

}  // extern "C"
