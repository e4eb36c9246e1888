// FP64-class products on the int8 tensor cores (tcgen05 kind::i8): the
// digit-slicing ("Ozaki") scheme.
//
// A row r of an FP64 operand is written as
//     a[r][k] = 2^e[r] * sum_{s=1..S} d_s[r][k] * 2^(-7 s)  (+ a remainder below 2^(e[r] - 7 S - 1))
// with balanced int8 digits d_s in [-64, 64] (e[r] makes max_k |a[r][k]| < 2^(e[r]-1)).
// A product of two sliced rows is then
//     sum_k a[r][k] b[c][k] = 2^(e_a[r] + e_b[c]) * sum_L 2^(-7 L) C_L[r][c],
//     C_L = sum_{p + q = L} sum_k d_p[r][k] d'_q[c][k]      (L = 2 .. S + 1)
// where every C_L is an exact int32 sum of int8 x int8 products (|C_L| <=
// S K 4096 < 2^31 for K <= 65536).  The S level sums of one output tile live
// in TMEM side by side; the epilogue combines them in FP64 (Horner in 2^-7),
// so the only rounding is the slicing remainder and the final FP64 additions:
// about 7 S - 1 significant bits per operand (S = 7: ~48 bits, S = 4: ~27).
//
// S(S+1)/2 int8 MMAs per K step replace one FP64 product; the int8 tensor
// cores run 2x the f16 rate (4.5 POPS dense on B200), against 40 TFLOP/s of
// FP64 FMA.
#pragma once

#include <cstdint>
#include <vector>

#include "kfb_internal.h"

namespace kfb {

constexpr int OZ_MAXS = 7;
constexpr int OZ_BM = 128;   // output rows per tile (TMEM lanes)
// output columns per tile (TMEM columns per level): S levels x BN <= 512
__host__ __device__ constexpr int oz_bn(int S) { return S <= 4 ? 128 : 64; }
constexpr int OZ_BK = 64;    // K bytes per pipeline stage (one 64-byte swizzle row)

// Sliced operand: S digit planes d[s][rows][kp] (kp a multiple of OZ_BK, the
// columns beyond K zero) and one exponent per row.
struct OzSlices {
    int8_t *d = nullptr;
    int *e = nullptr;
    int S = 0;
    long long rows = 0;
    int kp = 0;
};

inline int oz_kp(int k) { return (k + OZ_BK - 1) / OZ_BK * OZ_BK; }

// Slice rows of a row-major source: a[r][k] = src[r * ld + k] for r < rows,
// k < K.  Digits of columns K .. kp-1 are zero.
template <class T>
kfb_status oz_slice_rows(const T *src, long long rows, int K, long long ld, const OzSlices &out,
                         cudaStream_t s);
// Slice rows of a column-major source: a[r][k] = src[k * ld + r] (K <= 512).
kfb_status oz_slice_cols(const double *src, long long rows, int K, long long ld,
                         const OzSlices &out, cudaStream_t s);
// The same for any K (<= 65536): row maxima in a first pass (scratch_max, one
// 64-bit word per row), then the digits through shared-memory tiles.
kfb_status oz_slice_colmajor(const double *src, long long rows, int K, long long ld,
                             const OzSlices &out, unsigned long long *scratch_max,
                             cudaStream_t s);

// One output tile: rows a0 .. a0 + m - 1 of A against rows b0 .. b0 + n - 1 of
// B (m <= OZ_BM, n <= oz_bn(S)).  Output element (i, j) goes to
//     c[c_off + i * ldr + j * ldc]
// and, with lower != 0, only where a0 + i + lower_shift >= b0 + j.
struct OzTile {
    int a0, b0, m, n;
    long long c_off;
    int lower;
    int lower_shift;
};

// Epilogue: mode OZ_STORE c = alpha v, OZ_ADD c += alpha v.
enum OzMode : int { OZ_STORE = 0, OZ_ADD = 1 };
struct OzEpi {
    double *c = nullptr;
    long long ldr = 1, ldc = 0;
    int mode = OZ_STORE;
    double alpha = 1.0;
    const int *skip = nullptr;   // device flag: when non-zero the launch does nothing
    // one CTA per tile instead of one persistent CTA per SM: the SMs free up
    // tile by tile, so kernels of a higher-priority stream can start between
    // tiles (the Cholesky's look-ahead runs its bulk updates this way)
    int one_tile_per_cta = 0;
};

// C tiles = alpha * A . B^T (both operands sliced with the same S and kp).
// tiles: device array of ntiles OzTile.  err: device int raised when a
// pipeline wait times out (null: a private flag checked before returning,
// which synchronises the stream).
kfb_status oz_gemm(const OzSlices &A, const OzSlices &B, const OzTile *tiles, int ntiles,
                   const OzEpi &epi, int *err, cudaStream_t s);

// Tiles generated in the kernel instead of read from a list: the M x N
// product C[c_off + i ldr + j ldc] = alpha (A B^T)[i][j] (rows a_base + i of A,
// b_base + j of B), every tile of the rectangle (OZ_GEN_RECT) or only the
// tiles holding elements with i >= j, which are written alone (OZ_GEN_LOWER,
// a symmetric rank-K update of a lower triangle).
enum OzGenMode : int { OZ_GEN_RECT = 0, OZ_GEN_LOWER = 1 };
struct OzGen {
    int mode = OZ_GEN_RECT;
    int M = 0, N = 0;
    int a_base = 0, b_base = 0;
    long long c_off = 0;
};
int oz_gen_tiles(const OzGen &g, int S);
kfb_status oz_gemm_gen(const OzSlices &A, const OzSlices &B, const OzGen &g, const OzEpi &epi,
                       int *err, cudaStream_t s);

// Convenience: a dense product C (M x N) = alpha A B^T of two sliced operands,
// C[i * ldr + j * ldc] (tile list built and uploaded here).
kfb_status oz_gemm_dense(const OzSlices &A, const OzSlices &B, int M, int N, const OzEpi &epi,
                         cudaStream_t s);

#ifdef __CUDACC__
// Balanced base-128 digits of v = a 2^-e (|v| < 1/2): t = 128 v, d = rint(t),
// v = t - d, S times (every step exact in FP64; |d| <= 64).
template <int S>
__device__ __forceinline__ void oz_digits(double v, int8_t (&d)[S]) {
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const double t = v * 128.0;
        const double r = rint(t);
        d[s] = (int8_t)(int)r;
        v = t - r;
    }
}

// Row exponent e of a row with max |a| = amax: the smallest e with
// amax < 2^(e-1) (amax = m 2^x, m in [1, 2) -> e = x + 2), so |a 2^-e| < 1/2.
__device__ __forceinline__ int oz_row_exponent(double amax) {
    return amax > 0.0 ? ilogb(amax) + 2 : 0;
}

// x 2^p, exact: a multiplication by the power of two built from its exponent
// bits when 2^p is a normal double, ldexp otherwise.
__device__ __forceinline__ double oz_scale2(double x, int p) {
    if (p >= -1022 && p <= 1023) return x * __longlong_as_double((long long)(p + 1023) << 52);
    return ldexp(x, p);
}
#endif

}  // namespace kfb
