// Blocked Cholesky factorisation on the int8 tensor cores (chol.cu).
#pragma once

#include "kfb_internal.h"

namespace kfb {

// In-place A = L L^T of a dense symmetric n x n matrix in column-major storage
// with leading dimension ld; the lower triangle is read and overwritten with
// L (the strict upper triangle is not touched).  `slices` digit planes per
// operand for the tensor-core panel solves and trailing updates: 7 gives an
// FP64-class factor, 4 an FP32-class one (FP64 storage either way).  *info:
// 0, or the 1-based column of the first pivot that is not positive (as LAPACK
// potrf); the call synchronises the stream once, at the end.
kfb_status chol_dense(double *A, int n, long long ld, int slices, int *info, cudaStream_t s);

// Diagonal-block size of chol_dense.
constexpr int CHOL_NB = 128;

}  // namespace kfb
