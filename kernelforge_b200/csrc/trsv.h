// Triangular solves against a dense FP64 Cholesky factor (trsv.cu).
#pragma once

#include "kfb_internal.h"

namespace kfb {

// x = (L L^T)^{-1} b for the column-major lower factor L (n x n, leading
// dimension n).  prepare() inverts the 64 x 64 diagonal blocks (once per
// factor); solve() enqueues the two sweeps on s without synchronising;
// check() synchronises and reports a sweep whose bounded wait gave up.
struct TrsvPlan {
    int n = 0, nb = 0, grid = 0;
    DevBuf dinv, dinvt, sync;
    kfb_status prepare(const double *L, int n, cudaStream_t s);
    kfb_status solve(const double *L, const double *b, double *tmp, double *x, cudaStream_t s);
    kfb_status check(cudaStream_t s);
};

}  // namespace kfb
