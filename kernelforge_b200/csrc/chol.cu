// Blocked right-looking Cholesky factorisation with the panel solves and the
// trailing updates on the int8 tensor cores (digit-sliced FP64 products,
// ozaki.h).  Column-major storage, lower triangle.
//
// Per 128-column block j (c0 = 128 j, rows r0 = c0 + w .. n-1 below it):
//   1. chol_diag_kernel   one CTA factors the w x w diagonal block in shared
//                         memory (right-looking, one barrier per column) and
//                         records the first non-positive pivot;
//   2. chol_inv_kernel    W = L_jj^{-1}, one warp per column of W (a forward
//                         substitution with warp-wide dot products), 16 CTAs;
//   3. panel solve        L_21 = A_21 W^T: A_21 and W sliced into digit
//                         planes, one tensor-core product written over A_21;
//   4. trailing update    A_22 -= L_21 L_21^T on the lower triangle only
//                         (tiles generated in the GEMM kernel).
// The block order is that of LAPACK's right-looking dpotrf with the
// triangular solve replaced by a product with the inverted diagonal block (the
// inverse-based form used by GPU Cholesky codes, so that every O(n^3) part is
// a GEMM).  A failed pivot raises a device flag that makes every later kernel
// of the factorisation return at once; the host reads the pivot index once.
#include <algorithm>
#include <cmath>

#include "chol.h"
#include "ozaki.h"

namespace kfb {

namespace {

constexpr int NB = CHOL_NB;
constexpr int LDS = NB + 1;   // padded shared-memory column stride (doubles)
constexpr int DIAG_THREADS = 1024;
constexpr int INV_WARPS = 8;

// Factor the w x w block at (c0, c0) of the column-major matrix A in place.
__global__ void __launch_bounds__(DIAG_THREADS, 1)
    chol_diag_kernel(double *__restrict__ A, long long ld, int c0, int w, int *info, int *skip) {
    if (*(volatile int *)skip) return;
    extern __shared__ double t[];   // t[k * LDS + r] = A[c0 + r][c0 + k]
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double *blk = A + (long long)c0 * ld + c0;
    for (int idx = tid; idx < w * NB; idx += DIAG_THREADS) {
        const int k = idx / NB, r = idx - k * NB;
        if (r < w && r >= k) t[k * LDS + r] = blk[(long long)k * ld + r];
    }
    double dprev = 0.0;
    bool failed = false;
    for (int c = 0; c < w; ++c) {
        __syncthreads();
        const double acc = t[c * LDS + c];
        if (!(acc > 0.0) || !isfinite(acc)) {
            if (tid == 0) {
                *info = c0 + c + 1;
                atomicExch(skip, 1);
            }
            failed = true;
            break;
        }
        const double inv = 1.0 / acc;
        // column c - 1 is final: scale it (it is not read in this step)
        if (c > 0)
            for (int r = c + tid; r < w; r += DIAG_THREADS) t[(c - 1) * LDS + r] *= dprev;
        if (c > 0 && tid == 0) t[(c - 1) * LDS + (c - 1)] = 1.0 / dprev;
        // trailing update with the unscaled column c: A[r][k] -= A[r][c] A[k][c] / a_cc
        for (int k = c + 1 + wid; k < w; k += 32) {
            const double akc = t[c * LDS + k] * inv;
            for (int r = k + lane; r < w; r += 32) t[k * LDS + r] -= t[c * LDS + r] * akc;
        }
        dprev = rsqrt(acc);   // 1 / sqrt(a_cc)
    }
    if (failed) return;
    __syncthreads();
    for (int r = w - 1 + tid; r < w; r += DIAG_THREADS) t[(w - 1) * LDS + r] *= dprev;
    __syncthreads();
    if (tid == 0) t[(w - 1) * LDS + (w - 1)] = 1.0 / dprev;
    __syncthreads();
    for (int idx = tid; idx < w * NB; idx += DIAG_THREADS) {
        const int k = idx / NB, r = idx - k * NB;
        if (r < w && r >= k) blk[(long long)k * ld + r] = t[k * LDS + r];
    }
}

// W = L^{-1} of the factored w x w block (lower triangular), written
// column-major into W (ld NB, zero above the diagonal and beyond w).  Warp per
// column t: W[t][t] = 1 / L[t][t], W[r][t] = -(sum_{t<=k<r} L[r][k] W[k][t]) / L[r][r].
__global__ void __launch_bounds__(32 * INV_WARPS)
    chol_inv_kernel(const double *__restrict__ A, long long ld, int c0, int w,
                    double *__restrict__ W, const int *skip) {
    if (*(volatile const int *)skip) return;
    extern __shared__ double sm[];
    double *t = sm;                                  // [NB][LDS]: t[k * LDS + r] = L[r][k]
    double *wv = sm + NB * LDS;                      // [INV_WARPS][NB]
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const double *blk = A + (long long)c0 * ld + c0;
    for (int idx = tid; idx < w * NB; idx += blockDim.x) {
        const int k = idx / NB, r = idx - k * NB;
        if (r < w && r >= k) t[k * LDS + r] = blk[(long long)k * ld + r];
    }
    __syncthreads();
    const int col = blockIdx.x * INV_WARPS + wid;
    if (col >= NB) return;
    double *x = wv + wid * NB;
    double *out = W + (long long)col * NB;
    if (col >= w) {
        for (int r = lane; r < NB; r += 32) out[r] = 0.0;
        return;
    }
    for (int r = lane; r < NB; r += 32) x[r] = 0.0;
    __syncwarp();
    if (lane == 0) x[col] = 1.0 / t[col * LDS + col];
    __syncwarp();
    for (int r = col + 1; r < w; ++r) {
        double s = 0.0;
        for (int k = col + lane; k < r; k += 32) s += t[k * LDS + r] * x[k];
#pragma unroll
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) x[r] = -s / t[r * LDS + r];
        __syncwarp();
    }
    for (int r = lane; r < NB; r += 32) out[r] = x[r];
}

size_t diag_smem() { return (size_t)NB * LDS * sizeof(double); }
size_t inv_smem() { return (size_t)NB * LDS * sizeof(double) + (size_t)INV_WARPS * NB * 8; }

}  // namespace

kfb_status chol_dense(double *A, int n, long long ld, int slices, int *info, cudaStream_t s) {
    *info = 0;
    if (n <= 0) return KFB_OK;
    if (slices < 2 || slices > OZ_MAXS)
        return set_error(KFB_ERR_INVALID_ARG, "Cholesky digit planes %d outside 2..%d", slices,
                         OZ_MAXS);
    static bool attr = false;
    if (!attr) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(chol_diag_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)diag_smem()));
        KFB_CUDA_TRY(cudaFuncSetAttribute(chol_inv_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)inv_smem()));
        attr = true;
    }
    // flags: [0] info, [1] skip, [2] GEMM pipeline error
    DevBuf flags, Wd, psl, pex, wsl, wex;
    KFB_TRY(flags.alloc(4 * sizeof(int), s));
    KFB_TRY(zero(flags.ptr, 4 * sizeof(int), s));
    int *d_info = flags.as<int>(), *d_skip = d_info + 1, *d_err = d_info + 2;
    const int kp = NB;   // K of the panel products: one 128-column block
    const long long mmax = std::max(n - NB, 1);
    KFB_TRY(Wd.alloc((size_t)NB * NB * sizeof(double), s));
    KFB_TRY(psl.alloc((size_t)slices * mmax * kp, s));
    KFB_TRY(pex.alloc((size_t)mmax * sizeof(int), s));
    KFB_TRY(wsl.alloc((size_t)slices * NB * kp, s));
    KFB_TRY(wex.alloc((size_t)NB * sizeof(int), s));
    OzEpi epi;
    epi.c = A;
    epi.ldr = 1;
    epi.ldc = ld;
    epi.skip = d_skip;
    for (int c0 = 0; c0 < n; c0 += NB) {
        const int w = std::min(NB, n - c0);
        const int r0 = c0 + w, m = n - r0;
        chol_diag_kernel<<<1, DIAG_THREADS, diag_smem(), s>>>(A, ld, c0, w, d_info, d_skip);
        KFB_CUDA_TRY(cudaGetLastError());
        if (m == 0) break;
        chol_inv_kernel<<<NB / INV_WARPS, 32 * INV_WARPS, inv_smem(), s>>>(A, ld, c0, w,
                                                                         Wd.as<double>(), d_skip);
        KFB_CUDA_TRY(cudaGetLastError());
        OzSlices Wsl, P;
        Wsl.d = wsl.as<int8_t>();
        Wsl.e = wex.as<int>();
        Wsl.S = slices;
        Wsl.rows = w;
        Wsl.kp = kp;
        P.d = psl.as<int8_t>();
        P.e = pex.as<int>();
        P.S = slices;
        P.rows = m;
        P.kp = kp;
        double *a21 = A + (long long)c0 * ld + r0;
        KFB_TRY(oz_slice_cols(Wd.as<double>(), w, w, NB, Wsl, s));
        KFB_TRY(oz_slice_cols(a21, m, w, ld, P, s));
        // L21 = A21 W^T, written over A21
        OzGen g;
        g.mode = OZ_GEN_RECT;
        g.M = m;
        g.N = w;
        g.c_off = (long long)c0 * ld + r0;
        epi.mode = OZ_STORE;
        epi.alpha = 1.0;
        KFB_TRY(oz_gemm_gen(P, Wsl, g, epi, d_err, s));
        // A22 -= L21 L21^T (lower triangle)
        KFB_TRY(oz_slice_cols(a21, m, w, ld, P, s));
        g.mode = OZ_GEN_LOWER;
        g.M = m;
        g.N = m;
        g.c_off = (long long)r0 * ld + r0;
        epi.mode = OZ_ADD;
        epi.alpha = -1.0;
        KFB_TRY(oz_gemm_gen(P, P, g, epi, d_err, s));
    }
    int h[3] = {0, 0, 0};
    KFB_CUDA_TRY(cudaMemcpyAsync(h, d_info, 3 * sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (h[2]) return set_error(KFB_ERR_TIMEOUT, "Cholesky: a tensor-core pipeline wait timed out");
    *info = h[0];
    return KFB_OK;
}

}  // namespace kfb
