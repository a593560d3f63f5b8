// Test infrastructure only: a C-ABI shim over the reference's own CPU sources,
// compiled unmodified from the reference tree by oracle/Makefile into
// oracle/_ref/libbipp_ref.so. It is the parity pin for the restatement in
// oracle/bluebild.py and the CPU baseline timed by bench.py --impl reference.
// Nothing in the product (bipp_b200/) links or loads it.
//
// Wrapped reference entry points (paths relative to the reference project):
//   bipp::eigh_gram<T>            src/eigensolver.cpp:129-225
//   bipp::eigh<T>                 src/eigensolver.cpp:40-127
//   bipp::host::gram_matrix<T>    src/host/gram_matrix.cpp:29-64
//   bipp::host::virtual_vis<T>    src/host/virtual_vis.cpp:19-73
//   bipp::host::nuft_sum<T>       src/host/kernels/nuft_sum.cpp:9-31
//   bipp::host::DomainPartition   src/host/domain_partition.hpp:35-101 (grid)
#include <algorithm>
#include <complex>
#include <cstddef>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "bipp/bipp.hpp"
#include "bipp/exceptions.hpp"
#include "context_internal.hpp"
#include "host/domain_partition.hpp"
#include "host/gram_matrix.hpp"
#include "host/kernels/nuft_sum.hpp"
#include "host/virtual_vis.hpp"
#include "memory/allocator_factory.hpp"
#include "memory/view.hpp"

extern "C" void scipy_openblas_set_num_threads(int);
extern "C" int scipy_openblas_get_num_threads(void);

namespace {

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return 0;
  } catch (const bipp::GenericError& e) {
    return static_cast<int>(e.error_code());
  } catch (...) {
    return static_cast<int>(BIPP_GENERIC_ERROR);
  }
}

template <typename T>
int eigh_gram_t(T wl, std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* s,
                std::size_t lds, const std::complex<T>* w, std::size_t ldw, const T* xyz,
                std::size_t ldxyz, T* d, std::complex<T>* v, std::size_t ldv,
                std::size_t* nReduced, T* scale) {
  return guarded([&] {
    auto r = bipp::eigh_gram<T>(wl, nAntenna, nBeam, s, lds, w, ldw, xyz, ldxyz, d, v, ldv);
    *nReduced = r.first;
    *scale = r.second;
  });
}

template <typename T>
int eigh_t(T wl, std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* s,
           std::size_t lds, const std::complex<T>* w, std::size_t ldw, T* d,
           std::complex<T>* v, std::size_t ldv, std::size_t* nReduced, T* scale) {
  return guarded([&] {
    auto r = bipp::eigh<T>(wl, nAntenna, nBeam, s, lds, w, ldw, d, v, ldv);
    *nReduced = r.first;
    *scale = r.second;
  });
}

template <typename T>
int gram_t(std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* w, std::size_t ldw,
           const T* xyz, std::size_t ldxyz, T wl, std::complex<T>* g, std::size_t ldg) {
  return guarded([&] {
    std::shared_ptr<bipp::Allocator> alloc = bipp::AllocatorFactory::simple_host();
    bipp::ConstHostView<std::complex<T>, 2> wv(w, {nAntenna, nBeam}, {1, ldw});
    bipp::ConstHostView<T, 2> xv(xyz, {nAntenna, 3}, {1, ldxyz});
    bipp::HostView<std::complex<T>, 2> gv(g, {nBeam, nBeam}, {1, ldg});
    bipp::host::gram_matrix<T>(alloc, wv, xv, wl, gv);
  });
}

template <typename T>
int virtual_vis_t(T scale, std::size_t nAntenna, std::size_t nBeam, const T* d,
                  const std::complex<T>* v, std::size_t ldv, std::complex<T>* vv) {
  return guarded([&] {
    bipp::ContextInternal ctx(BIPP_PU_CPU);
    bipp::ConstHostView<T, 1> dv(d, nBeam, 1);
    bipp::ConstHostView<std::complex<T>, 2> vview(v, {nAntenna, nBeam}, {1, ldv});
    bipp::HostView<std::complex<T>, 1> out(vv, nAntenna * nAntenna, 1);
    bipp::host::virtual_vis<T>(ctx, scale, dv, vview, out);
  });
}

// The reference direct sum is single threaded; the harness splits the output
// points over host threads (each thread calls the reference function on a
// disjoint output range), so the CPU baseline uses every core.
template <typename T>
int nuft_sum_t(T alpha, std::size_t nIn, const std::complex<T>* input, const T* u, const T* v,
               const T* w, std::size_t nOut, const T* x, const T* y, const T* z, T* out,
               int nThreads) {
  return guarded([&] {
    if (nThreads <= 1 || nOut < 2) {
      bipp::host::nuft_sum<T>(alpha, nIn, input, u, v, w, nOut, x, y, z, out);
      return;
    }
    const std::size_t nt = std::min<std::size_t>(nThreads, nOut);
    const std::size_t chunk = (nOut + nt - 1) / nt;
    std::vector<std::thread> pool;
    for (std::size_t t = 0; t < nt; ++t) {
      const std::size_t b = t * chunk;
      if (b >= nOut) break;
      const std::size_t n = std::min(chunk, nOut - b);
      pool.emplace_back([=] {
        bipp::host::nuft_sum<T>(alpha, nIn, input, u, v, w, n, x + b, y + b, z + b, out + b);
      });
    }
    for (auto& th : pool) th.join();
  });
}

template <typename T>
int partition_grid_t(const std::size_t* dims, std::size_t n, const T* x, const T* y, const T* z,
                     std::size_t* permutOut, std::size_t* groupBegin, std::size_t* groupSize) {
  return guarded([&] {
    std::shared_ptr<bipp::Allocator> alloc = bipp::AllocatorFactory::simple_host();
    std::array<std::size_t, 3> gd = {dims[0], dims[1], dims[2]};
    auto part = bipp::host::DomainPartition::grid<T, 3>(
        alloc, gd,
        {bipp::ConstHostView<T, 1>(x, n, 1), bipp::ConstHostView<T, 1>(y, n, 1),
         bipp::ConstHostView<T, 1>(z, n, 1)});
    const auto& groups = part.groups();
    for (std::size_t g = 0; g < groups.size(); ++g) {
      groupBegin[g] = groups[g].begin;
      groupSize[g] = groups[g].size;
    }
    // recover the permutation by applying it to the identity sequence
    std::vector<std::size_t> idx(n), outIdx(n);
    for (std::size_t i = 0; i < n; ++i) idx[i] = i;
    part.template apply<std::size_t, std::size_t>(bipp::ConstHostView<std::size_t, 1>(idx.data(), n, 1),
                                         bipp::HostView<std::size_t, 1>(outIdx.data(), n, 1));
    // outIdx[permut[i]] = i  -> permut[i] = position of element i
    for (std::size_t p = 0; p < n; ++p) permutOut[outIdx[p]] = p;
  });
}

}  // namespace

#pragma GCC visibility push(default)
extern "C" {

void ref_set_threads(int n) { scipy_openblas_set_num_threads(n); }
int ref_get_threads(void) { return scipy_openblas_get_num_threads(); }

int ref_eigh_gram_f32(float wl, std::size_t nA, std::size_t nB, const void* s, std::size_t lds,
                      const void* w, std::size_t ldw, const float* xyz, std::size_t ldxyz,
                      float* d, void* v, std::size_t ldv, std::size_t* nRed, float* scale) {
  return eigh_gram_t<float>(wl, nA, nB, static_cast<const std::complex<float>*>(s), lds,
                            static_cast<const std::complex<float>*>(w), ldw, xyz, ldxyz, d,
                            static_cast<std::complex<float>*>(v), ldv, nRed, scale);
}
int ref_eigh_gram_f64(double wl, std::size_t nA, std::size_t nB, const void* s, std::size_t lds,
                      const void* w, std::size_t ldw, const double* xyz, std::size_t ldxyz,
                      double* d, void* v, std::size_t ldv, std::size_t* nRed, double* scale) {
  return eigh_gram_t<double>(wl, nA, nB, static_cast<const std::complex<double>*>(s), lds,
                             static_cast<const std::complex<double>*>(w), ldw, xyz, ldxyz, d,
                             static_cast<std::complex<double>*>(v), ldv, nRed, scale);
}
int ref_eigh_f32(float wl, std::size_t nA, std::size_t nB, const void* s, std::size_t lds,
                 const void* w, std::size_t ldw, float* d, void* v, std::size_t ldv,
                 std::size_t* nRed, float* scale) {
  return eigh_t<float>(wl, nA, nB, static_cast<const std::complex<float>*>(s), lds,
                       static_cast<const std::complex<float>*>(w), ldw, d,
                       static_cast<std::complex<float>*>(v), ldv, nRed, scale);
}
int ref_eigh_f64(double wl, std::size_t nA, std::size_t nB, const void* s, std::size_t lds,
                 const void* w, std::size_t ldw, double* d, void* v, std::size_t ldv,
                 std::size_t* nRed, double* scale) {
  return eigh_t<double>(wl, nA, nB, static_cast<const std::complex<double>*>(s), lds,
                        static_cast<const std::complex<double>*>(w), ldw, d,
                        static_cast<std::complex<double>*>(v), ldv, nRed, scale);
}
int ref_gram_matrix_f32(std::size_t nA, std::size_t nB, const void* w, std::size_t ldw,
                        const float* xyz, std::size_t ldxyz, float wl, void* g, std::size_t ldg) {
  return gram_t<float>(nA, nB, static_cast<const std::complex<float>*>(w), ldw, xyz, ldxyz, wl,
                       static_cast<std::complex<float>*>(g), ldg);
}
int ref_gram_matrix_f64(std::size_t nA, std::size_t nB, const void* w, std::size_t ldw,
                        const double* xyz, std::size_t ldxyz, double wl, void* g,
                        std::size_t ldg) {
  return gram_t<double>(nA, nB, static_cast<const std::complex<double>*>(w), ldw, xyz, ldxyz, wl,
                        static_cast<std::complex<double>*>(g), ldg);
}
int ref_virtual_vis_f32(float scale, std::size_t nA, std::size_t nB, const float* d,
                        const void* v, std::size_t ldv, void* vv) {
  return virtual_vis_t<float>(scale, nA, nB, d, static_cast<const std::complex<float>*>(v), ldv,
                              static_cast<std::complex<float>*>(vv));
}
int ref_virtual_vis_f64(double scale, std::size_t nA, std::size_t nB, const double* d,
                        const void* v, std::size_t ldv, void* vv) {
  return virtual_vis_t<double>(scale, nA, nB, d, static_cast<const std::complex<double>*>(v),
                               ldv, static_cast<std::complex<double>*>(vv));
}
int ref_nuft_sum_f32(float alpha, std::size_t nIn, const void* input, const float* u,
                     const float* v, const float* w, std::size_t nOut, const float* x,
                     const float* y, const float* z, float* out, int nThreads) {
  return nuft_sum_t<float>(alpha, nIn, static_cast<const std::complex<float>*>(input), u, v, w,
                           nOut, x, y, z, out, nThreads);
}
int ref_nuft_sum_f64(double alpha, std::size_t nIn, const void* input, const double* u,
                     const double* v, const double* w, std::size_t nOut, const double* x,
                     const double* y, const double* z, double* out, int nThreads) {
  return nuft_sum_t<double>(alpha, nIn, static_cast<const std::complex<double>*>(input), u, v, w,
                            nOut, x, y, z, out, nThreads);
}
int ref_partition_grid_f32(const std::size_t* dims, std::size_t n, const float* x,
                           const float* y, const float* z, std::size_t* permut,
                           std::size_t* groupBegin, std::size_t* groupSize) {
  return partition_grid_t<float>(dims, n, x, y, z, permut, groupBegin, groupSize);
}
int ref_partition_grid_f64(const std::size_t* dims, std::size_t n, const double* x,
                           const double* y, const double* z, std::size_t* permut,
                           std::size_t* groupBegin, std::size_t* groupSize) {
  return partition_grid_t<double>(dims, n, x, y, z, permut, groupBegin, groupSize);
}

}  // extern "C"
#pragma GCC visibility pop
