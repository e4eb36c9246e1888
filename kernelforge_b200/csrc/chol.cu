// Blocked right-looking Cholesky factorisation: the diagonal blocks and panel
// solves on the FP64 CUDA cores, the trailing updates on the int8 tensor cores
// (digit-sliced FP64 products, ozaki.h).  Column-major storage, lower triangle.
//
// Two levels of blocking.  Outer panels of 512 columns; inside one, per
// 128-column block j (c0 = 128 j, rows r0 = c0 + w .. n-1 below it):
//   1. chol_block_kernel  one CTA factors the w x w diagonal block in shared
//                         memory in 32-column sub-blocks (a warp factors each
//                         32 x 32 diagonal sub-block in registers, then inverts
//                         it; the CTA solves the rows below and updates the
//                         rest of the block), then forms W = L_jj^{-1} by
//                         block substitution; the first non-positive pivot is
//                         recorded (LAPACK potrf's info);
//   2. chol_panel_kernel  L_21 = A_21 W^T in FP64 (64 rows per CTA, W and the
//                         rows staged in shared memory by cp.async), written
//                         over A_21, together with the digit planes and row
//                         exponents of L_21;
//   3. inner update       the outer panel's remaining columns (all rows below
//                         them) -= L_21 L_21^T, K = 128 (tensor cores);
// then, once per outer panel, the panel is sliced again (one row scale over
// its 512 columns) and everything right of it is updated by tensor-core
// products with K = 512 on the lower triangle only: the next outer panel's
// columns on a high-priority stream, the rest on a low-priority stream with one
// CTA per tile, so that the next panel's diagonal blocks, panels and inner
// updates run while that bulk update proceeds (look-ahead; the digit planes of
// consecutive outer panels alternate between two buffers).  The FP64 read-modify-write
// of the trailing matrix, the memory cost of a right-looking factorisation,
// thereby happens once per 512 columns instead of once per 128.
// The block order is that of LAPACK's right-looking dpotrf with the panel's
// triangular solve replaced by a product with the inverted diagonal block
// (the inverse-based form used by GPU Cholesky codes).  A failed pivot raises
// a device flag that makes every later kernel of the factorisation return at
// once; the host reads the pivot index once, at the end.
#include <algorithm>
#include <cmath>

#include "chol.h"
#include "ozaki.h"

namespace kfb {

namespace {

constexpr int NB = CHOL_NB;       // 128
constexpr int SB = 32;            // sub-block of the diagonal factorisation
constexpr int LDT = NB + 2;       // shared column stride of the block (doubles; even)
constexpr int LDW = SB + 1;       // shared column stride of a 32 x 32 inverse block
constexpr int NWB = 10;           // lower 32 x 32 blocks of a 128 x 128 triangle
constexpr int BLK_THREADS = 512;
constexpr int BLK_WARPS = BLK_THREADS / 32;
constexpr int NB2 = 4 * NB;       // outer panel (two-level blocking)
constexpr int PR = 64;            // panel rows per CTA
constexpr int PANEL_THREADS = 256;

static_assert(NB == 4 * SB, "the block kernel assumes four sub-blocks");

__host__ __device__ constexpr int wblk(int i, int j) { return i * (i + 1) / 2 + j; }

template <class F>
constexpr size_t blk_smem() {
    return ((size_t)NB * LDT + (size_t)NWB * SB * LDW + SB) * sizeof(F) + 16;
}
constexpr size_t PANEL_SMEM = ((size_t)NB * NB + (size_t)NB * (PR + 1)) * sizeof(double);

// Asynchronous global -> shared copies (cp.async): `bytes` of 8 or 16, with
// the shared destination zero-filled instead when `valid` is false (the
// source pointer must still be a valid address).
__device__ __forceinline__ void cp_async(void *sdst, const void *gsrc, int bytes, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(sdst));
    if (bytes == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc),
                     "r"(valid ? 16 : 0)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(gsrc),
                     "r"(valid ? 8 : 0)
                     : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}

constexpr unsigned FULL = 0xffffffffu;

// 1 / sqrt(d) for the pivots: the FP32 estimate refined by two Newton steps in
// FP64 (each squares the relative error: 2^-23 -> 2^-46 -> below FP64
// rounding), which is shorter on the pivot chain than the FP64 library
// routine; outside the FP32 range the library routine.
__device__ __forceinline__ double pivot_rsqrt(double d) {
    if (!(d > 1e-30 && d < 1e30)) return rsqrt(d);
    double r = (double)rsqrtf((float)d);
    const double hd = 0.5 * d;
    r = r * fma(-hd * r, r, 1.5);
    r = r * fma(-hd * r, r, 1.5);
    return r;
}
__device__ __forceinline__ float pivot_rsqrt(float d) { return rsqrtf(d); }

template <class F> struct Vec2;
template <> struct Vec2<double> { using type = double2; };
template <> struct Vec2<float> { using type = float2; };

// Factor the w x w block at (c0, c0) of the column-major matrix A in place
// (lower triangle) and write W = L^{-1} column-major into Wout (NB x NB, zero
// above the diagonal and beyond w), with the arithmetic in F: double for an
// FP64-class factor, float for an FP32-class one (the FP32 pivot chain is
// several times shorter: one-instruction shuffles, rsqrt, FMAs).
//
// Shared memory: T[k * LDT + r] = A[c0 + r][c0 + k] (zero outside the lower
// w x w triangle); WB holds the lower 32 x 32 blocks of W, block (i, j) at
// WB + wblk(i, j) * SB * LDW, element (r, c) at [c * LDW + r]; rd[r] = 1 /
// L[o + r][o + r] of the current sub-block.
template <class F>
__global__ void __launch_bounds__(BLK_THREADS, 1)
    chol_block_kernel(double *__restrict__ A, long long ld, int c0, int w,
                      double *__restrict__ Wout, int *info, int *skip) {
    using F2 = typename Vec2<F>::type;
    if (*(volatile int *)skip) return;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    F *T = reinterpret_cast<F *>(sm_raw);
    F *WB = T + NB * LDT;
    F *rd = WB + NWB * SB * LDW;   // 1 / L[o + r][o + r] of the current sub-block
    int *flag = reinterpret_cast<int *>(rd + SB);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const double *blk = A + (long long)c0 * ld + c0;
    if constexpr (sizeof(F) == 8) {
        if (w == NB && (ld & 1) == 0 && (c0 & 1) == 0) {
            // a full block, 16-byte aligned rows: pairs of rows per copy (the
            // strict upper triangle comes along and is never read)
#pragma unroll 4
            for (int idx = tid; idx < NB * NB / 2; idx += BLK_THREADS) {
                const int k = idx / (NB / 2), r = 2 * (idx - k * (NB / 2));
                cp_async(T + k * LDT + r, blk + (long long)k * ld + r, 16, true);
            }
        } else {
#pragma unroll 4
            for (int idx = tid; idx < NB * NB; idx += BLK_THREADS) {
                const int k = idx / NB, r = idx - k * NB;
                const bool v = r < w && k < w && r >= k;
                cp_async(T + k * LDT + r, v ? blk + (long long)k * ld + r : blk, 8, v);
            }
        }
        cp_async_wait_all();
    } else {
        // eight independent loads in flight per thread, then the conversions
        constexpr int PER = NB * NB / BLK_THREADS;
        static_assert(PER % 8 == 0, "load batches");
        for (int b = 0; b < PER; b += 8) {
            double v[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = tid + (b + u) * BLK_THREADS, k = idx / NB, r = idx - k * NB;
                v[u] = (r < w && k < w && r >= k) ? blk[(long long)k * ld + r] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = tid + (b + u) * BLK_THREADS, k = idx / NB, r = idx - k * NB;
                T[k * LDT + r] = (F)v[u];
            }
        }
    }
    if (tid == 0) *flag = 0;
    __syncthreads();
    const int P = (w + SB - 1) / SB;
    for (int p = 0; p < P; ++p) {
        const int o = p * SB, wp = min(SB, w - o);
        if (warp == 0) {
            // (a) right-looking factorisation of the wp x wp diagonal
            // sub-block in registers: lane = row, a[k] = L[lane][k] (k <= lane)
            F a[SB];
#pragma unroll
            for (int k = 0; k < SB; ++k) a[k] = (k <= lane) ? T[(o + k) * LDT + o + lane] : F(0);
            F rinv = F(0);   // 1 / L[lane][lane]
            int bad = SB;        // first column with a non-positive pivot
#pragma unroll
            for (int c = 0; c < SB; ++c) {
                if (c < wp) {
                    const F d = __shfl_sync(FULL, a[c], c);
                    if (!(d > F(0)) || !isfinite(d)) bad = min(bad, c);   // warp-uniform
                    const F rs = pivot_rsqrt(d);
                    const F l = (lane == c) ? d * rs : a[c] * rs;
                    if (lane == c) rinv = rs;
                    a[c] = l;
                    // the scaled column is final: write it, then read it back as
                    // a broadcast (faster than 31 shuffles on the pivot chain:
                    // 164 vs 247 cycles per column in FP32, 420 vs 523 in FP64)
                    if (lane >= c && lane < wp) T[(o + c) * LDT + o + lane] = l;
                    __syncwarp();
#pragma unroll
                    for (int k = c + 1; k < SB; ++k) {
                        const F lk = T[(o + c) * LDT + o + k];   // L[k][c] (0 beyond wp)
                        if constexpr (sizeof(F) == 4) {
                            // FP32: a select and an unconditional FMA (no
                            // divergent branch per k: 71 -> 60 us per block)
                            const F m = (k <= lane) ? l : F(0);
                            a[k] = fma(-m, lk, a[k]);
                        } else {
                            // FP64: the masked FMAs would cost more than the branch
                            if (k <= lane) a[k] = fma(-l, lk, a[k]);
                        }
                    }
                }
            }
            if (bad < wp) {
                if (lane == 0) {
                    *info = c0 + o + bad + 1;
                    atomicExch(skip, 1);
                    *flag = 1;
                }
            } else {
                rd[lane] = rinv;
            }
        }
        __syncthreads();
        if (*flag) return;   // block-uniform after the barrier
        if (warp == 0) {
            // (b) W_pp = L_pp^{-1}, lane = column l, forward substitution in
            // right-looking order: W[r][l] = s[r] / L[r][r], then
            // s[r'] -= L[r'][r] W[r][l] for r' > r (column r of L read as a
            // broadcast), so each row adds one FMA and one multiply to the
            // dependent chain instead of a dot product
            F sacc[SB];
#pragma unroll
            for (int r = 0; r < SB; ++r) sacc[r] = (r == lane) ? F(1) : F(0);
            F *Wp = WB + wblk(p, p) * SB * LDW + lane * LDW;
#pragma unroll
            for (int r = 0; r < SB; ++r) {
                const F xr = (r < wp && lane < wp) ? sacc[r] * rd[r] : F(0);
                Wp[r] = xr;
#pragma unroll
                for (int r2 = r + 1; r2 < SB; ++r2)
                    sacc[r2] = fma(-T[(o + r) * LDT + o + r2], xr, sacc[r2]);
            }
        }
        __syncthreads();
        const int rb = o + wp, mr = w - rb;
        if (mr <= 0) continue;
        const int ns = (mr + 31) / 32;
        // (c) rows below the sub-block: X[r][c] = sum_{k <= c} A[r][o + k] W_pp[c][k]
        //     (unit = 32 rows x 8 columns; lane = row)
        {
            const F *Wp = WB + wblk(p, p) * SB * LDW;
            const int u = warp, s = u >> 2, g = u & 3;
            const int r = rb + 32 * s + lane;
            const bool act = s < ns && r < w;
            F x[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) x[j] = F(0);
            if (s < ns) {
                const int rr = min(r, NB - 1);
#pragma unroll
                for (int k = 0; k < SB; ++k) {
                    const F a = T[(o + k) * LDT + rr];
#pragma unroll
                    for (int j = 0; j < 8; ++j) x[j] = fma(a, Wp[k * LDW + 8 * g + j], x[j]);
                }
            }
            __syncthreads();
            if (act)
#pragma unroll
                for (int j = 0; j < 8; ++j) T[(o + 8 * g + j) * LDT + r] = x[j];
            __syncthreads();
        }
        // (d) the rest of the block: T[k][r] -= sum_c X[r][c] X[k][c], rb <= k <= r < w
        //     (unit = 32 rows of strip s x 8 columns; strip s has 4 (s + 1) groups)
        {
            const int nunits = 2 * ns * (ns + 1);
            for (int u = warp; u < nunits; u += BLK_WARPS) {
                int s = 0;
                while (2 * (s + 1) * (s + 2) <= u) ++s;
                const int g = u - 2 * s * (s + 1);
                const int r = rb + 32 * s + lane, k0 = rb + 8 * g;
                const int rr = min(r, NB - 1);
                F acc[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) acc[j] = F(0);
#pragma unroll
                for (int c = 0; c < SB; ++c) {
                    const F *col = T + (o + c) * LDT;
                    const F a = col[rr];
                    const F2 *kv = reinterpret_cast<const F2 *>(col + k0);
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const F2 b = kv[j];
                        acc[2 * j] = fma(a, b.x, acc[2 * j]);
                        acc[2 * j + 1] = fma(a, b.y, acc[2 * j + 1]);
                    }
                }
                if (r < w)
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                        if (k0 + j <= r) T[(k0 + j) * LDT + r] -= acc[j];
            }
            __syncthreads();
        }
    }
    // W = L^{-1} off the diagonal, by block substitution along block diagonals
    // d = i - j:  M = sum_{j <= k < i} L_ik W_kj,  W_ij = -W_ii M
    // (unit = one 8-column group of one block pair; lane = row)
    for (int d = 1; d < P; ++d) {
        const int nunits = 4 * (P - d);
        for (int u = warp; u < nunits; u += BLK_WARPS) {
            const int j = u >> 2, g = u & 3, i = j + d;
            F m[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) m[q] = F(0);
            for (int k = j; k < i; ++k) {
                const F *Wkj = WB + wblk(k, j) * SB * LDW;
#pragma unroll
                for (int t = 0; t < SB; ++t) {
                    const F l = T[(SB * k + t) * LDT + SB * i + lane];
#pragma unroll
                    for (int q = 0; q < 8; ++q) m[q] = fma(l, Wkj[(8 * g + q) * LDW + t], m[q]);
                }
            }
            F *Wij = WB + wblk(i, j) * SB * LDW;
#pragma unroll
            for (int q = 0; q < 8; ++q) Wij[(8 * g + q) * LDW + lane] = m[q];
        }
        __syncthreads();
        for (int u = warp; u < nunits; u += BLK_WARPS) {
            const int j = u >> 2, g = u & 3, i = j + d;
            const F *Wii = WB + wblk(i, i) * SB * LDW;
            F *Wij = WB + wblk(i, j) * SB * LDW;
            F o[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) o[q] = F(0);
#pragma unroll
            for (int t = 0; t < SB; ++t) {
                const F wv = Wii[t * LDW + lane];
#pragma unroll
                for (int q = 0; q < 8; ++q) o[q] = fma(wv, Wij[(8 * g + q) * LDW + t], o[q]);
            }
            // only this warp reads its columns of M: overwrite them in place
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 8; ++q) Wij[(8 * g + q) * LDW + lane] = -o[q];
        }
        __syncthreads();
    }
    double *ablk = A + (long long)c0 * ld + c0;
    for (int idx = tid; idx < w * NB; idx += BLK_THREADS) {
        const int k = idx / NB, r = idx - k * NB;
        if (r < w && r >= k) ablk[(long long)k * ld + r] = (double)T[k * LDT + r];
    }
    // W column-major, two rows per 16-byte store
    for (int idx = tid; idx < NB * NB / 2; idx += BLK_THREADS) {
        const int c = idx / (NB / 2), r = 2 * (idx - c * (NB / 2));
        double v[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int rr = r + u;
            v[u] = (rr < w && c < w && rr >= c)
                       ? (double)WB[wblk(rr / SB, c / SB) * SB * LDW + (c % SB) * LDW + (rr % SB)]
                       : 0.0;
        }
        reinterpret_cast<double2 *>(Wout)[idx] = make_double2(v[0], v[1]);
    }
}

// L_21 = A_21 W^T for rows r0 + 64 blockIdx.x ... of the panel (column c0 ..
// c0 + 127), written over A_21, plus the S digit planes d[s][row][k] (kp =
// NB) and row exponents of L_21 for the tensor-core trailing update.
//
// Shared memory: Ws[k * NB + c] = W[c][k] (= Wout, column-major W); Xs[k *
// (PR + 1) + r] = A[row r][c0 + k], then the rows of L_21.
template <int S>
__global__ void __launch_bounds__(PANEL_THREADS)
    chol_panel_kernel(double *__restrict__ A, long long ld, int c0, int r0, int m,
                      const double *__restrict__ Wout, int8_t *__restrict__ dpl,
                      int *__restrict__ dex, const int *skip) {
    if (*(volatile const int *)skip) return;
    extern __shared__ __align__(16) double sm[];
    double *Ws = sm;
    double *Xs = sm + NB * NB;
    constexpr int LDX = PR + 1;
    const int tid = threadIdx.x;
    const int rbase = blockIdx.x * PR;
#pragma unroll 8
    for (int idx = tid; idx < NB * NB / 2; idx += PANEL_THREADS)
        cp_async(Ws + 2 * idx, Wout + 2 * idx, 16, true);
    const double *arows = A + (long long)c0 * ld + r0 + rbase;
#pragma unroll 8
    for (int idx = tid; idx < NB * PR; idx += PANEL_THREADS) {
        const int k = idx / PR, r = idx - k * PR;
        const bool v = rbase + r < m;
        cp_async(Xs + k * LDX + r, v ? arows + (long long)k * ld + r : arows, 8, v);
    }
    cp_async_wait_all();
    __syncthreads();
    // thread tile: rows 4 rg .. 4 rg + 3, columns 8 cg .. 8 cg + 7
    const int rg = tid & 15, cg = tid >> 4;
    double acc[4][8];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
    const int kmax = 8 * cg + 8;   // W[c][k] = 0 for k > c
    for (int k = 0; k < kmax; ++k) {
        double a[4], b[8];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = Xs[k * LDX + 4 * rg + i];
        const double2 *wv = reinterpret_cast<const double2 *>(Ws + k * NB + 8 * cg);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const double2 t = wv[j];
            b[2 * j] = t.x;
            b[2 * j + 1] = t.y;
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) Xs[(8 * cg + j) * LDX + 4 * rg + i] = acc[i][j];
    __syncthreads();
    for (int idx = tid; idx < NB * PR; idx += PANEL_THREADS) {
        const int c = idx / PR, r = idx - c * PR;
        if (rbase + r < m) A[(long long)(c0 + c) * ld + r0 + rbase + r] = Xs[c * LDX + r];
    }
    // digit planes: a warp per row, lane l holds columns l, l + 32, l + 64, l + 96
    const int warp = tid >> 5, lane = tid & 31;
    const long long plane = (long long)m * NB;
    for (int rl = warp; rl < PR; rl += PANEL_THREADS / 32) {
        const int row = rbase + rl;
        if (row >= m) break;
        double v[4], mx = 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            v[q] = Xs[(lane + 32 * q) * LDX + rl];
            mx = fmax(mx, fabs(v[q]));
        }
#pragma unroll
        for (int o = 16; o; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        const int ex = oz_row_exponent(mx);
        if (lane == 0) dex[row] = ex;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            int8_t dg[S];
            oz_digits<S>(ldexp(v[q], -ex), dg);
#pragma unroll
            for (int s = 0; s < S; ++s) dpl[s * plane + (long long)row * NB + lane + 32 * q] = dg[s];
        }
    }
}

template <int S>
kfb_status launch_panel(double *A, long long ld, int c0, int r0, int m, const double *W,
                        int8_t *dpl, int *dex, const int *skip, cudaStream_t s) {
    static bool attr = false;
    if (!attr) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(chol_panel_kernel<S>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)PANEL_SMEM));
        attr = true;
    }
    chol_panel_kernel<S><<<(m + PR - 1) / PR, PANEL_THREADS, PANEL_SMEM, s>>>(A, ld, c0, r0, m, W,
                                                                             dpl, dex, skip);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

kfb_status panel(int S, double *A, long long ld, int c0, int r0, int m, const double *W,
                 int8_t *dpl, int *dex, const int *skip, cudaStream_t s) {
    switch (S) {
        case 2: return launch_panel<2>(A, ld, c0, r0, m, W, dpl, dex, skip, s);
        case 3: return launch_panel<3>(A, ld, c0, r0, m, W, dpl, dex, skip, s);
        case 4: return launch_panel<4>(A, ld, c0, r0, m, W, dpl, dex, skip, s);
        case 5: return launch_panel<5>(A, ld, c0, r0, m, W, dpl, dex, skip, s);
        case 6: return launch_panel<6>(A, ld, c0, r0, m, W, dpl, dex, skip, s);
        case 7: return launch_panel<7>(A, ld, c0, r0, m, W, dpl, dex, skip, s);
        default: return set_error(KFB_ERR_INVALID_ARG, "digit planes S=%d", S);
    }
}

}  // namespace

namespace {

// The two streams of the look-ahead, per device: the critical path (diagonal
// blocks, panels, the updates the next panel waits for) at the highest
// priority, the bulk trailing updates at the lowest.
struct CholStreams {
    cudaStream_t crit = nullptr, bulk = nullptr;
};

kfb_status chol_streams(CholStreams *&out) {
    static CholStreams per_dev[16];
    int dev = 0;
    KFB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16) return set_error(KFB_ERR_UNSUPPORTED, "device index %d", dev);
    CholStreams &cs = per_dev[dev];
    if (!cs.crit) {
        int least = 0, greatest = 0;
        KFB_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        KFB_CUDA_TRY(cudaStreamCreateWithPriority(&cs.crit, cudaStreamNonBlocking, greatest));
        KFB_CUDA_TRY(cudaStreamCreateWithPriority(&cs.bulk, cudaStreamNonBlocking, least));
    }
    out = &cs;
    return KFB_OK;
}

// Events of one factorisation, destroyed with it.
struct CholEvents {
    cudaEvent_t ev[6] = {};
    kfb_status init() {
        for (auto &e : ev) KFB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        return KFB_OK;
    }
    ~CholEvents() {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    }
};

}  // namespace

kfb_status chol_dense(double *A, int n, long long ld, int slices, int *info, cudaStream_t s) {
    *info = 0;
    if (n <= 0) return KFB_OK;
    if (slices < 2 || slices > OZ_MAXS)
        return set_error(KFB_ERR_INVALID_ARG, "Cholesky digit planes %d outside 2..%d", slices,
                         OZ_MAXS);
    static bool attr = false;
    if (!attr) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(chol_block_kernel<double>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)blk_smem<double>()));
        KFB_CUDA_TRY(cudaFuncSetAttribute(chol_block_kernel<float>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)blk_smem<float>()));
        attr = true;
    }
    // the diagonal blocks in FP32 for an FP32-class factor (4 or fewer planes)
    const bool f32blk = slices <= 4;
    CholStreams *cs = nullptr;
    KFB_TRY(chol_streams(cs));
    const cudaStream_t sc = cs->crit, sb = cs->bulk;
    CholEvents E;
    KFB_TRY(E.init());
    cudaEvent_t ev_start = E.ev[0], ev_slice = E.ev[1], ev_bulk = E.ev[2], ev_crit_end = E.ev[3],
                ev_bulk_end = E.ev[4];
    // everything below is ordered after the caller's work on s
    KFB_CUDA_TRY(cudaEventRecord(ev_start, s));
    KFB_CUDA_TRY(cudaStreamWaitEvent(sc, ev_start, 0));
    KFB_CUDA_TRY(cudaStreamWaitEvent(sb, ev_start, 0));
    // flags: [0] info, [1] skip, [2] GEMM pipeline error
    DevBuf flags, Wd, psl, pex, osl[2], oex[2];
    KFB_TRY(flags.alloc(4 * sizeof(int), sc));
    KFB_TRY(zero(flags.ptr, 4 * sizeof(int), sc));
    int *d_info = flags.as<int>(), *d_skip = d_info + 1, *d_err = d_info + 2;
    const long long mmax = std::max(n - NB, 1);
    KFB_TRY(Wd.alloc((size_t)NB * NB * sizeof(double), sc));
    KFB_TRY(psl.alloc((size_t)slices * mmax * NB, sc));
    KFB_TRY(pex.alloc((size_t)mmax * sizeof(int), sc));
    if (n > NB2)
        for (int b = 0; b < 2; ++b) {
            KFB_TRY(osl[b].alloc((size_t)slices * (n - NB2) * NB2, sc));
            KFB_TRY(oex[b].alloc((size_t)(n - NB2) * sizeof(int), sc));
        }
    // on an early (error) return, let both streams finish before the buffers
    // above are released (destroyed after this guard)
    struct Drain {
        cudaStream_t a, b;
        bool armed = true;
        ~Drain() {
            if (armed) {
                cudaStreamSynchronize(a);
                cudaStreamSynchronize(b);
            }
        }
    } drain{sc, sb};
    // the bulk stream's first work reads buffers allocated on the critical one
    KFB_CUDA_TRY(cudaEventRecord(ev_slice, sc));
    KFB_CUDA_TRY(cudaStreamWaitEvent(sb, ev_slice, 0));
    OzEpi epi;
    epi.c = A;
    epi.ldr = 1;
    epi.ldc = ld;
    epi.skip = d_skip;
    epi.mode = OZ_ADD;
    epi.alpha = -1.0;
    OzEpi epi_bulk = epi;
    epi_bulk.one_tile_per_cta = 1;
    bool bulk_pending = false;   // a bulk update was enqueued and not waited for
    for (int o0 = 0, P = 0; o0 < n; o0 += NB2, ++P) {
        const int ow = std::min(NB2, n - o0);   // outer panel: columns o0 .. o0 + ow - 1
        for (int c0 = o0; c0 < o0 + ow; c0 += NB) {
            const int w = std::min(NB, n - c0);
            const int r0 = c0 + w, m = n - r0;
            if (f32blk)
                chol_block_kernel<float><<<1, BLK_THREADS, blk_smem<float>(), sc>>>(
                    A, ld, c0, w, Wd.as<double>(), d_info, d_skip);
            else
                chol_block_kernel<double><<<1, BLK_THREADS, blk_smem<double>(), sc>>>(
                    A, ld, c0, w, Wd.as<double>(), d_info, d_skip);
            KFB_CUDA_TRY(cudaGetLastError());
            if (m == 0) break;
            // L21 = A21 W^T and its digit planes
            KFB_TRY(panel(slices, A, ld, c0, r0, m, Wd.as<double>(), psl.as<int8_t>(),
                          pex.as<int>(), d_skip, sc));
            // the rest of the outer panel: columns r0 .. o0 + ow - 1, every row
            // below them, -= L21 L21^T (a lower trapezoid)
            const int nin = o0 + ow - r0;
            if (nin > 0) {
                OzSlices Pl;
                Pl.d = psl.as<int8_t>();
                Pl.e = pex.as<int>();
                Pl.S = slices;
                Pl.rows = m;
                Pl.kp = NB;
                OzGen g;
                g.mode = OZ_GEN_LOWER;
                g.M = m;
                g.N = nin;
                g.c_off = (long long)r0 * ld + r0;
                KFB_TRY(oz_gemm_gen(Pl, Pl, g, epi, d_err, sc));
            }
        }
        // everything right of the outer panel -= L_panel L_panel^T (K = ow, the
        // panel sliced once more with one row scale over its columns), in two
        // parts: the next outer panel's columns on the critical stream (the
        // next panel's blocks wait for them), the rest on the bulk stream,
        // where it overlaps the next panel's blocks, panels and inner updates
        const int R = o0 + ow, M = n - R;
        if (M <= 0) continue;
        OzSlices O;
        O.d = osl[P & 1].as<int8_t>();
        O.e = oex[P & 1].as<int>();
        O.S = slices;
        O.rows = M;
        O.kp = oz_kp(ow);
        KFB_TRY(oz_slice_cols(A + (long long)o0 * ld + R, M, ow, ld, O, sc));
        KFB_CUDA_TRY(cudaEventRecord(ev_slice, sc));
        // the previous bulk update wrote these columns too: wait for it
        if (bulk_pending) KFB_CUDA_TRY(cudaStreamWaitEvent(sc, ev_bulk, 0));
        const int na = std::min(NB2, M);
        OzGen ga;
        ga.mode = OZ_GEN_LOWER;
        ga.M = M;
        ga.N = na;
        ga.c_off = (long long)R * ld + R;
        KFB_TRY(oz_gemm_gen(O, O, ga, epi, d_err, sc));
        if (M > na) {
            KFB_CUDA_TRY(cudaStreamWaitEvent(sb, ev_slice, 0));
            OzGen gb;
            gb.mode = OZ_GEN_LOWER;
            gb.M = M - na;
            gb.N = M - na;
            gb.a_base = na;
            gb.b_base = na;
            gb.c_off = (long long)(R + na) * ld + (R + na);
            KFB_TRY(oz_gemm_gen(O, O, gb, epi_bulk, d_err, sb));
            KFB_CUDA_TRY(cudaEventRecord(ev_bulk, sb));
            bulk_pending = true;
        } else {
            bulk_pending = false;
        }
    }
    // join both streams back into the caller's
    KFB_CUDA_TRY(cudaEventRecord(ev_crit_end, sc));
    KFB_CUDA_TRY(cudaEventRecord(ev_bulk_end, sb));
    KFB_CUDA_TRY(cudaStreamWaitEvent(s, ev_crit_end, 0));
    KFB_CUDA_TRY(cudaStreamWaitEvent(s, ev_bulk_end, 0));
    int h[3] = {0, 0, 0};
    KFB_CUDA_TRY(cudaMemcpyAsync(h, d_info, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    drain.armed = false;   // both streams joined into s, which is idle now
    if (h[2]) return set_error(KFB_ERR_TIMEOUT, "Cholesky: a tensor-core pipeline wait timed out");
    *info = h[0];
    return KFB_OK;
}

}  // namespace kfb
