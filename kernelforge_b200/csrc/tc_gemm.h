// Grouped tensor-core GEMM (tc_gemm.cu): C = A . B^T over problems that are
// row blocks / column windows of two K-major fp16 (or bf16) 2-D arrays.
#pragma once

#include <cuda_fp16.h>

#include <vector>

#include "derivs.h"

namespace kfb {

// One K-major operand array (rows x cols elements, 16-bit), split pair or not.
struct TcOperand {
    const void *hi = nullptr;
    const void *lo = nullptr;  // only with 3 products
    long long rows = 0, cols = 0;
};

// C[row_off + m][col_off + n] = alpha * sum_k A[a_row0 + m][a_k0 + k] B[b_row0 + n][b_k0 + k]
// for m < M, n < N, k < K (K a multiple of 16, a_k0 / b_k0 multiples of 8).
struct TcProb {
    int a_row0, a_k0, b_row0, b_k0;
    int M, N, K;
    int row_off, col_off;
    int diag;
    double alpha;
};

struct TcTile {
    int prob, m0, n0, pad;
};

// nprod = 3: split operands, hi*hi + hi*lo + lo*hi; nprod = 1: hi only.
kfb_status tc_gemm_grouped(const TcOperand &A, const TcOperand &B, int nprod, bool bf16,
                           const std::vector<TcProb> &probs, const ElemSink &sink,
                           cudaStream_t s);

// Split packers: multiply by a power-of-two scale (returned in *scale; the
// largest magnitude lands near 2^14) and write the fp16 pair hi = fp16(v),
// lo = fp16(v - hi).  GEMM results are divided by the two operands' scales.
template <class T>
kfb_status split_rows(const T *src, long long n, __half *hi, __half *lo, float *scale,
                      cudaStream_t s);
template <class T>
kfb_status transpose_split_dx(const T *dx, int nm, int ma, int rep, __half *hi, __half *lo,
                              float *scale, cudaStream_t s);
template <class T>
kfb_status transpose_split_y(const T *Y, int np, int ma1, int rep, int ld, __half *hi,
                             __half *lo, float *scale, cudaStream_t s);

}  // namespace kfb
