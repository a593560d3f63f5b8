// NUFFT engine shared by the collect/get plan and the batched pipeline.
#pragma once

#include <cufft.h>

#include <map>
#include <vector>

#include "common.cuh"
#include "context.hpp"
#include "fft_kernels.cuh"
#include "nufft_kernels.cuh"

namespace bippb200 {

// Pixel lattice fitted to the pixel coordinates (l, m): l = l0 + a Al + b Bl,
// m = m0 + a Am + b Bm, pixel index p = a Nb + b.
struct Lattice {
  bool ok = false;
  int Na = 0, Nb = 0;
  double l0 = 0, m0 = 0, Al = 0, Bl = 0, Am = 0, Bm = 0;
  double maxResidL = 0, maxResidM = 0;  // max |l - lattice|, |m - lattice|
};

Lattice fit_lattice(const std::vector<double>& l, const std::vector<double>& m);

// ES kernel width and shape for a tolerance at upsampling factor 2 (as used by type-1/3
// NUFFTs with the "exponential of semicircle" kernel).
// fine-grid oversampling in x, y and w: the tuning table's nufft.grid_per_1024 / 1024
constexpr int kMaxPipelineLevels = 8;  // energy levels of one pipeline (NUFFT channels)
void es_params(double eps, double sigma, int& W, float& beta);

class NufftCore {
public:
  // Pixel side: lattice + per-pixel n (FP64). nch = channels per transform.
  void setup(bipp_ctx_s* ctx, const Lattice& lat, const std::vector<double>& n, double eps, int nch,
             const std::vector<double>* dl = nullptr, const std::vector<double>* dm = nullptr, double su = 1.0,
             double sv = 1.0, int levels = 0);

  // Per transform: w-range of the points (already scaled to phase units).
  void begin(double wmin, double wmax);
  // Per transform (after begin): enable the first-order lattice-residual channels and
  // the u/v normalisation of their values.
  void set_corr(bool on, double su, double sv);
  int* counts() { return counts_.get<int>(); }
  // After the count kernels: scan -> offsets & cursor; allocate records for nPoints
  void end_count(long long nPoints);
  int* cursor() { return cursor_.get<int>(); }
  PtRec* records() { return rec_.get<PtRec>(); }
  // values of the sorted points, [point][channel] (channels() per point)
  float2* values() { return vals_.get<float2>(); }
  // capacity in points of records() / values() (the scatter kernels' bounds guard)
  long long value_stride() const { return valStride_; }
  // per-channel accumulator of zero-baseline values (added to every pixel)
  double* zero_acc() { return zeroAcc_.get<double>(); }
  // spread/FFT/w-sum over all slabs and accumulate Re(...) into image[ch][P] (ld P)
  void execute(float* image, long long ldImage, double* stageMs = nullptr);

  const NufftGeom& geom() const { return g_; }
  // statistics of the last execute(): points spread, slabs (spreading launches), bytes of
  // grid written by the spreading (all slabs), work items, tiles split into several
  // parts (more points than the spread.items_cap tunable; their parts accumulate with atomics)
  long long lastPoints = 0, lastSlabs = 0, lastGridBytes = 0, lastItems = 0, lastSplitTiles = 0;
  long long num_pixels() const { return (long long)g_.Na * g_.Nb; }
  int channels() const { return nch_; }
  bool sincos64() const { return eps_ < 1e-6; }
  double su() const { return su_; }
  double sv() const { return sv_; }
  bool corr_terms() const { return corrTerms_; }

private:
  bipp_ctx_s* ctx_ = nullptr;
  NufftGeom g_{};
  int nch_ = 1, levels_ = 1;
  double eps_ = 1e-5;
  double Sn_ = 0;
  bool corrTerms_ = false, corrCapable_ = false;
  double su_ = 1, sv_ = 1;
  long long nkeys_ = 0, valStride_ = 0;
  DevBuf nTilde_, decon_, dl_, dm_, counts_, offsets_, cursor_, blockSums_, rec_, vals_, grid_, acc_;
  DevBuf itemKeys_, itemsAlt_, sortTmp_, workCounters_;
  DevBuf qz_, qw_, zeroAcc_, load_, items_, errFlag_, splitCount_, parts_, itemOff_, itemSums_, clearFlag_, clearOff_, clearList_;
  DevBuf valScale_;   // per-channel value scale of the FP16 spreader operands
  // batched 2-D cuFFT plans by batch size (channels x slab planes), for grid sizes without
  // a compiled pruned-FFT plan or nufft.fft = 0
  std::map<int, cufftHandle> plans_;
  // pruned two-pass inverse FFT (rows along x, then the kept columns along y) and its
  // twiddle tables (nx entries for the rows, then ny for the columns)
  FftLinePlan rowPlan_{}, colPlan_{};
  FftLinesKernel rowKernel_ = nullptr, colKernel_ = nullptr;
  bool fftPlansOk_ = false;
  DevBuf fftTw_;
  int slabTiles_ = 1;
  // inverse 2-D FFT of the first planesUsed planes of every channel of the slab: pruned
  // (cell (a, b) of a plane then holds pixel (a, b)'s output) or in full by cuFFT
  void inverse_fft(int slabPlanes, int planesUsed, float2* slab, bool pruned);
  void exclusive_scan(const int* in, int* out, long long n);

public:
  ~NufftCore();
};

// Staging of one sample of a collect/get plan (bipp_nufft_create) in device memory: the
// caller writes the sample's scaled uvw at nufft_stage_uvw (three coordinate arrays of
// nBaselines floats, ld nufft_stage_ld) and the values of image im at
// nufft_stage_values(plan, im) (nBaselines complex floats) on the plan's stream, then
// nufft_commit adds the sample (transforming the batch when it is full), as
// bipp_nufft_add_s does for host arrays.
float* nufft_stage_uvw(bipp_nufft_t p);
float2* nufft_stage_values(bipp_nufft_t p, size_t im);
long long nufft_stage_ld(bipp_nufft_t p);
void nufft_commit(bipp_nufft_t p);

// Gauss-Legendre nodes/weights on [-1, 1]
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w);

}  // namespace bippb200
