// Exception types of the bipp C++ API. The class names, hierarchy and error codes are
// those of the reference (include/bipp/exceptions.hpp:16-140) so that callers' handlers
// keep working; each carries the message reported by the library.
#pragma once

#include <bipp/config.h>
#include <bipp/errors.h>

#include <stdexcept>
#include <string>

namespace bipp {

class BIPP_EXPORT GenericError : public std::runtime_error {
public:
  GenericError() : std::runtime_error("BIPP: Generic error") {}
  explicit GenericError(const std::string& msg) : std::runtime_error(msg) {}
  virtual BippError error_code() const noexcept { return BIPP_GENERIC_ERROR; }
};

#define BIPP_B200_ERROR_CLASS(NAME, BASE, CODE, DEFAULT_MSG)                      \
  class BIPP_EXPORT NAME : public BASE {                                          \
  public:                                                                         \
    NAME() : BASE(DEFAULT_MSG) {}                                                 \
    explicit NAME(const std::string& msg) : BASE(msg) {}                          \
    BippError error_code() const noexcept override { return CODE; }               \
  };

BIPP_B200_ERROR_CLASS(InternalError, GenericError, BIPP_INTERNAL_ERROR, "BIPP: Internal error")
BIPP_B200_ERROR_CLASS(InvalidParameterError, GenericError, BIPP_INVALID_PARAMETER_ERROR, "BIPP: InvalidParameterError error")
BIPP_B200_ERROR_CLASS(InvalidPointerError, GenericError, BIPP_INVALID_POINTER_ERROR, "BIPP: InvalidPointerError error")
BIPP_B200_ERROR_CLASS(InvalidAllocatorFunctionError, GenericError, BIPP_INVALID_ALLOCATOR_FUNCTION,
                      "BIPP: InvalidAllocatorFunctionError error")
BIPP_B200_ERROR_CLASS(EigensolverError, GenericError, BIPP_EIGENSOLVER_ERROR, "BIPP: EigensolverError error")
BIPP_B200_ERROR_CLASS(HDF5Error, GenericError, BIPP_HDF5_ERROR, "BIPP: HDF5Error error")
BIPP_B200_ERROR_CLASS(NotImplementedError, GenericError, BIPP_NOT_IMPLEMENTED_ERROR, "BIPP: NotImplementedError error")
BIPP_B200_ERROR_CLASS(GPUError, GenericError, BIPP_GPU_ERROR, "BIPP: GPU Error")
BIPP_B200_ERROR_CLASS(GPUSupportError, GPUError, BIPP_GPU_SUPPORT_ERROR, "BIPP: Not compiled with GPU support")
BIPP_B200_ERROR_CLASS(GPUBlasError, GPUError, BIPP_GPU_BLAS_ERROR, "BIPP: GPU BLAS error")
BIPP_B200_ERROR_CLASS(MPIError, GPUError, BIPP_MPI_ERROR, "BIPP: MPI Error")
BIPP_B200_ERROR_CLASS(FileError, GenericError, BIPP_FILE_ERROR, "BIPP: FileError")

#undef BIPP_B200_ERROR_CLASS

}  // namespace bipp
