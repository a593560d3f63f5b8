/* Error codes of the bipp C/C++ API. Enumerators and values follow the reference
 * (include/bipp/errors.h:5-66) so that existing error handling keeps working. */
#pragma once

enum BippError {
  BIPP_SUCCESS,
  BIPP_GENERIC_ERROR,
  BIPP_INTERNAL_ERROR,
  BIPP_INVALID_PARAMETER_ERROR,
  BIPP_INVALID_POINTER_ERROR,
  BIPP_INVALID_HANDLE_ERROR,
  BIPP_EIGENSOLVER_ERROR,
  BIPP_NOT_IMPLEMENTED_ERROR,
  BIPP_GPU_ERROR,
  BIPP_GPU_SUPPORT_ERROR,
  BIPP_GPU_BLAS_ERROR,
  BIPP_INVALID_ALLOCATOR_FUNCTION,
  BIPP_MPI_ERROR,
  BIPP_HDF5_ERROR,
  BIPP_FILE_ERROR
};

#ifndef __cplusplus
typedef enum BippError BippError;
#endif
