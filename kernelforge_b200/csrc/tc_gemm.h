// Grouped tensor-core GEMM (tc_gemm.cu): C = A . B^T over problems that are
// row blocks / column windows of two K-major fp16 (or bf16) 2-D arrays.
#pragma once

#include <cuda_bf16.h>
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

// Epilogue of the grouped GEMM.  EPI_SINK writes alpha * acc through the
// ElemSink.  The other modes serve the feature-map kernels; (row, col) is the
// global position (row_off + m, col_off + n) and z = alpha * acc + bias[col]
// (bias optional):
//   EPI_DENSE      zf32[row * ld + col] = z  (or += z, atomically, with accumulate)
//                  act[row * ld + col] = bf16(cos z)       (optional)
//                  act_t[col * ld_t + row] = bf16(cos z)   (optional)
//   EPI_DSIN_T     act_t[col * ld_t + row] = bf16(-alpha * acc * sin(aux[row * ld + col]))
//                  (back-propagation through a cos activation)
//   EPI_COS_MOLSUM molsum[mol[row] * ld + col] += scale * cos z, each run of
//                  rows of one molecule summed before its atomic add
//   EPI_SIN_RUNSUM molsum[mol[row] * ld + col] +=
//                      scale * sin(aux[atom[row] * ld_aux + col]) * alpha * acc,
//                  runs of rows with one destination summed as above
//   EPI_YSPLIT     the Hessian's Y in the layout its contraction reads: problem
//                  row m = (c, k) = (m / y_rep, m % y_rep), column n ->
//                  (p, i) = ymap[b_row0 + n] (p < 0: skipped), and the fp16 pair
//                  of alpha * acc goes to yhi / ylo[((p y_ld2 + c) y_ma1 + i) y_rep + k]
//                  (y_rep % 8 == 0, yhi / ylo 16-byte aligned)
enum TcEpiMode : int {
    EPI_SINK = 0,
    EPI_DENSE = 1,
    EPI_DSIN_T = 2,
    EPI_COS_MOLSUM = 3,
    EPI_SIN_RUNSUM = 4,
    EPI_YSPLIT = 5
};

struct TcEpi {
    int mode = EPI_SINK;
    int tile_n64 = 0;  // 128 x 64 tiles (problems with N <= 64 waste no MMA columns)
    int sink_t = 0;    // EPI_SINK: alpha * acc stored at (col, row) instead of (row, col)
    int vec = 0;         // set by tc_gemm_grouped: 16-byte row stores allowed
    int accumulate = 0;  // EPI_DENSE: zf32 += z (atomic; split-K problems)
    float *zf32 = nullptr;
    __nv_bfloat16 *act = nullptr;
    __nv_bfloat16 *act_t = nullptr;
    const float *aux = nullptr;
    const float *bias = nullptr;
    const int *mol = nullptr;
    const int *atom = nullptr;  // EPI_SIN_RUNSUM: row of aux for each output row
    float *molsum = nullptr;
    long long ld = 0, ld_t = 0, ld_aux = 0;
    float scale = 1.f;
    const int2 *ymap = nullptr;   // EPI_YSPLIT
    __half *yhi = nullptr, *ylo = nullptr;
    int y_rep = 0, y_ma1 = 0, y_ld2 = 0;
};

// nprod = 3: split operands, hi*hi + hi*lo + lo*hi; nprod = 1: hi only.
// err_flag: null = wait for the kernel and report a pipeline timeout now;
// otherwise the kernel raises *err_flag (device int) and the call returns
// without synchronising (the caller checks the flag later).
kfb_status tc_gemm_grouped(const TcOperand &A, const TcOperand &B, int nprod, bool bf16,
                           const std::vector<TcProb> &probs, const ElemSink &sink,
                           cudaStream_t s, const TcEpi &epi = TcEpi(), int *err_flag = nullptr);

// Split packers: multiply by a power-of-two scale (returned in *scale; the
// largest magnitude of the entries the GEMMs read lands near 2^14) and write
// the fp16 pair hi = fp16(v), lo = fp16(v - hi).  GEMM results are divided by
// the two operands' scales.
//   split_rows:         every entry of src is read;
//   transpose_split_dx: nat (device int32, per molecule) limits the scale to
//                       the real atoms, padding may hold anything; 32 x 32
//                       tiles wholly beyond the real atoms stay unwritten;
//   transpose_split_y:  amax (device float) is the largest |entry| the
//                       producer wrote (the rest of Y is never read).
template <class T>
kfb_status split_rows(const T *src, long long n, __half *hi, __half *lo, float *scale,
                      cudaStream_t s);
// Jr[(m, j, c)][k] = dX[m][j][k][c] as scaled fp16 pairs: a K-major row of rep
// per (atom, coordinate column); rows of padding atoms and columns are not
// written.  blockmap (device, per atom m * ma + j, optional) moves atom (m, j)'s
// 3 ma rows to block blockmap[m * ma + j] (< 0: not written).
template <class T>
kfb_status transpose_split_dx_rows(const T *dx, int nm, int ma, int rep, const int *nat,
                                   __half *hi, __half *lo, float *scale, cudaStream_t s,
                                   const int *blockmap = nullptr);
template <class T>
kfb_status transpose_split_dx(const T *dx, int nm, int ma, int rep, const int *nat, __half *hi,
                              __half *lo, float *scale, cudaStream_t s);
// Host copy of a power of two that brings the device float *dmax to about
// 2^14 (synchronises the stream).
kfb_status pow2_from_device(const float *dmax, cudaStream_t s, float *scale);
template <class T>
kfb_status transpose_split_y(const T *Y, int np, int ma1, int rep, int ld, const float *amax,
                             __half *hi, __half *lo, float *scale, cudaStream_t s);

}  // namespace kfb
