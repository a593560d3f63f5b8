// Build configuration used when the reference's own CPU sources are compiled
// as the parity oracle: host BLAS/LAPACK through the C interfaces, no GPU, no MPI.
#pragma once
#define BIPP_BLAS_C
#define BIPP_LAPACK_C
#define BIPP_VERSION "1.0.0-oracle"
#include <bipp/bipp_export.h>
