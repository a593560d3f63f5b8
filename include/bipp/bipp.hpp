// Eigensolver entry points of the bipp C++ API (reference: include/bipp/bipp.hpp:47-75).
// Same templates and argument meaning; both run on the GPU through the B200 library
// (a process-wide default context is used, as the reference functions take none).
#pragma once

#include <bipp/communicator.hpp>
#include <bipp/config.h>
#include <bipp/context.hpp>
#include <bipp/dataset.hpp>
#include <bipp/enums.h>
#include <bipp/exceptions.hpp>
#include <bipp/image_data.hpp>
#include <bipp/image_prop.hpp>
#include <bipp/image_synthesis.hpp>

#include <complex>
#include <cstddef>
#include <type_traits>
#include <utility>

namespace bipp {

template <typename T, typename = std::enable_if_t<std::is_same_v<T, double> || std::is_same_v<T, float>>>
BIPP_EXPORT auto eigh(T wl, std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* s, std::size_t lds,
                      const std::complex<T>* w, std::size_t ldw, T* d, std::complex<T>* v, std::size_t ldv)
    -> std::pair<std::size_t, T>;

template <typename T, typename = std::enable_if_t<std::is_same_v<T, double> || std::is_same_v<T, float>>>
BIPP_EXPORT auto eigh_gram(T wl, std::size_t nAntenna, std::size_t nBeam, const std::complex<T>* s, std::size_t lds,
                           const std::complex<T>* w, std::size_t ldw, const T* xyz, std::size_t ldxyz, T* d,
                           std::complex<T>* v, std::size_t ldv) -> std::pair<std::size_t, T>;

}  // namespace bipp
