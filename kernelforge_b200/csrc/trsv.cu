// Triangular solves with one right-hand side against a dense FP64 Cholesky
// factor (column-major lower L, leading dimension n): x = (L L^T)^{-1} b as
// L t = b, then L^T x = t.  This is the preconditioner application of the
// refinement loop of the KRR solve; the library call it replaces
// (potrs -> two trsm with one column) walks the factor in dependent column
// panels and ran at about a quarter of the factor's read bandwidth.
//
// Design (64-row blocks, nb = ceil(n / 64)):
//  * the 64 x 64 diagonal blocks are inverted once per factor (block per
//    diagonal block, thread per column), so the solve of a block is a
//    matrix-vector product instead of 64 dependent steps;
//  * one persistent cooperative kernel per direction; block I is owned by CTA
//    I mod grid.  Its CTA accumulates the off-diagonal tiles against the
//    solution blocks as they are published and then applies the inverted
//    diagonal block.  Blocks finish in solve order (block I needs block I-1),
//    so publication is a single counter `done` (st.release / ld.acquire at
//    gpu scope) and a CTA stages every block published so far in one batch;
//  * every wait is bounded: after TRSV_WAIT_LIMIT polls the CTA raises *err
//    and all CTAs leave; the host reads *err once per solve sequence.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels_common.cuh"
#include "trsv.h"

namespace kfb {

namespace {

constexpr int TB = 64;                  // rows per block
constexpr int TB_BATCH = 8;             // solution blocks staged per wait
constexpr int TRSV_THREADS = 256;       // 64 rows x 4 column groups
constexpr unsigned long long TRSV_WAIT_NS = 1000000000ull;   // one second of %globaltimer

__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned long long trsv_clock_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Thread 0: wait until more than `need` blocks are published; returns the
// published count, or -1 when the wait gave up (or another CTA gave up).  The
// limit is elapsed time on %globaltimer (one second), not a poll count:
// __nanosleep is only a hint, so a count would not bound the wait's length.
__device__ int wait_published(const int *done, int need, int *err) {
    const unsigned long long t0 = trsv_clock_ns();
    while (true) {
        const int d = ld_acquire(done);
        if (d > need) return d;
        if (*reinterpret_cast<volatile int *>(err)) return -1;
        if (trsv_clock_ns() - t0 > TRSV_WAIT_NS) break;
        __nanosleep(32);
    }
    atomicExch(err, 1);
    return -1;
}

// Inverse of each 64 x 64 lower diagonal block: dinv[I] column-major
// (dinv[I][r + 64 c] = (L_II^{-1})[r][c]) and dinvt[I] its transpose;
// rows/columns beyond n are the identity.
__global__ void __launch_bounds__(TB) trsv_dinv_kernel(const double *__restrict__ L, int n,
                                                      double *__restrict__ dinv,
                                                      double *__restrict__ dinvt) {
    __shared__ double a[TB][TB + 1];   // a[r][c] = L_II[r][c]
    const int I = blockIdx.x, i0 = I * TB, m = min(TB, n - i0);
    const int c = threadIdx.x;
    for (int r = 0; r < TB; ++r)
        a[r][c] = (r < m && c < m && r >= c) ? L[(size_t)(i0 + r) + (size_t)(i0 + c) * n] : 0.0;
    __syncthreads();
    // column c of the inverse by forward substitution on e_c, kept in dinv
    double *zc = dinv + (size_t)I * TB * TB + (size_t)TB * c;
    for (int r = 0; r < TB; ++r) zc[r] = (r == c && c >= m) ? 1.0 : 0.0;
    if (c < m) {
        zc[c] = 1.0 / a[c][c];
        for (int r = c + 1; r < m; ++r) {
            double s = 0.0;
            for (int j = c; j < r; ++j) s = fma(a[r][j], zc[j], s);
            zc[r] = -s / a[r][r];
        }
    }
    __syncthreads();
    const double *d = dinv + (size_t)I * TB * TB;
    double *dt = dinvt + (size_t)I * TB * TB;
    for (int r = 0; r < TB; ++r) dt[r + TB * c] = d[c + TB * r];   // transpose
}

// L t = b.  Thread (r = t & 63, g = t >> 6) accumulates row r over the
// columns c = g, g + 4, ... of each tile.  Before its first wait a CTA issues
// the loads of what the critical step needs (the inverted diagonal block into
// shared memory, the tile of the block just before it into registers), so
// that once block I-1 is published only x_{I-1} is fetched.
__global__ void __launch_bounds__(TRSV_THREADS) trsv_lower_kernel(
    const double *__restrict__ L, int n, int nb, const double *__restrict__ dinv,
    const double *__restrict__ b, double *t_out, int *done, int *err) {
    __shared__ double xs[TB_BATCH * TB];
    __shared__ double red[4][TB];
    __shared__ double dsm[TB * TB];
    __shared__ int avail;
    const int t = threadIdx.x, r = t & (TB - 1), g = t >> 6;
    for (int I = blockIdx.x; I < nb; I += gridDim.x) {
        const int i0 = I * TB, row = i0 + r;
        const bool rv = row < n;
        __syncthreads();   // dsm of the previous block consumed
        for (int e = t; e < TB * TB; e += TRSV_THREADS) dsm[e] = dinv[(size_t)I * TB * TB + e];
        double lvl[TB / 4];   // tile (I, I-1)
#pragma unroll
        for (int k = 0; k < TB / 4; ++k)
            lvl[k] = (rv && I > 0) ? L[(size_t)row + (size_t)((I - 1) * TB + g + 4 * k) * n] : 0.0;
        double acc = 0.0;
        for (int J = 0; J < I;) {
            if (t == 0) avail = wait_published(done, J, err);
            __syncthreads();
            const int d = avail;
            if (d < 0) return;
            const int J1 = min(min(d, I), J + TB_BATCH);
            for (int e = t; e < (J1 - J) * TB; e += TRSV_THREADS)
                xs[e] = __ldcg(t_out + (size_t)J * TB + e);   // published blocks: < i0 <= n
            __syncthreads();
            for (int jj = J; jj < J1; ++jj) {
                const double *xv = xs + (jj - J) * TB;
                if (jj == I - 1) {
#pragma unroll
                    for (int k = 0; k < TB / 4; ++k) acc = fma(lvl[k], xv[g + 4 * k], acc);
                    continue;
                }
                const double *col = L + (size_t)row + (size_t)jj * TB * n;
                double lv[TB / 4];
#pragma unroll
                for (int k = 0; k < TB / 4; ++k)
                    lv[k] = rv ? col[(size_t)(g + 4 * k) * n] : 0.0;
#pragma unroll
                for (int k = 0; k < TB / 4; ++k) acc = fma(lv[k], xv[g + 4 * k], acc);
            }
            __syncthreads();   // xs consumed
            J = J1;
        }
        red[g][r] = acc;
        __syncthreads();
        if (t < TB) xs[t] = rv ? b[row] - (red[0][t] + red[1][t] + red[2][t] + red[3][t]) : 0.0;
        __syncthreads();
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < TB / 4; ++k) s = fma(dsm[r + TB * (g + 4 * k)], xs[g + 4 * k], s);
        __syncthreads();   // red reused
        red[g][r] = s;
        __syncthreads();
        if (t < TB && rv) {
            t_out[row] = red[0][t] + red[1][t] + red[2][t] + red[3][t];
            __threadfence();
        }
        __syncthreads();
        if (t == 0) st_release(done, I + 1);
    }
}

// L^T x = t, blocks in reverse order (rank q = nb - 1 - I is the publication
// order).  Thread (r, g) accumulates, for the columns c = g, g + 4, ... of
// block I, L[j0 + r][i0 + c] x[j0 + r] over the later blocks J; the row
// partials of each column are summed by warp shuffles and across the two
// warps of a column group.  Prefetches as in the forward sweep (tile of block
// I+1, the transposed inverse of the diagonal block).
__global__ void __launch_bounds__(TRSV_THREADS) trsv_upper_kernel(
    const double *__restrict__ L, int n, int nb, const double *__restrict__ dinvt,
    const double *__restrict__ tv, double *x, int *done, int *err) {
    __shared__ double xs[TB_BATCH * TB];
    __shared__ double red[2][TB];   // [half of the rows][column]
    __shared__ double dsm[TB * TB];
    __shared__ int avail;
    const int t = threadIdx.x, r = t & (TB - 1), g = t >> 6;
    const int lane = t & 31, half = r >> 5;
    for (int q = blockIdx.x; q < nb; q += gridDim.x) {
        const int I = nb - 1 - q, i0 = I * TB;
        __syncthreads();   // dsm of the previous block consumed
        for (int e = t; e < TB * TB; e += TRSV_THREADS) dsm[e] = dinvt[(size_t)I * TB * TB + e];
        double lvl[TB / 4];   // tile (I+1, I)
        {
            const int j = (I + 1) * TB + r;
            const bool jv = q > 0 && j < n;
#pragma unroll
            for (int k = 0; k < TB / 4; ++k)
                lvl[k] = jv ? L[(size_t)j + (size_t)(i0 + g + 4 * k) * n] : 0.0;
        }
        double acc[TB / 4];
#pragma unroll
        for (int k = 0; k < TB / 4; ++k) acc[k] = 0.0;
        // later blocks J = nb - 1 - p for published ranks p < q
        for (int p = 0; p < q;) {
            if (t == 0) avail = wait_published(done, p, err);
            __syncthreads();
            const int d = avail;
            if (d < 0) return;
            const int p1 = min(min(d, q), p + TB_BATCH);
            // stage blocks J = nb-1-p .. nb-p1 (rank order)
            for (int e = t; e < (p1 - p) * TB; e += TRSV_THREADS) {
                const int pp = p + e / TB, rr = e % TB;
                const int j = (nb - 1 - pp) * TB + rr;
                xs[e] = j < n ? __ldcg(x + j) : 0.0;
            }
            __syncthreads();
            for (int pp = p; pp < p1; ++pp) {
                const double xr = xs[(pp - p) * TB + r];
                if (pp == q - 1) {   // block I+1
#pragma unroll
                    for (int k = 0; k < TB / 4; ++k) acc[k] = fma(lvl[k], xr, acc[k]);
                    continue;
                }
                const int j = (nb - 1 - pp) * TB + r;
                const bool jv = j < n;
                const double *rowp = L + (size_t)j + (size_t)i0 * n;
                double lv[TB / 4];
#pragma unroll
                for (int k = 0; k < TB / 4; ++k) lv[k] = jv ? rowp[(size_t)(g + 4 * k) * n] : 0.0;
#pragma unroll
                for (int k = 0; k < TB / 4; ++k) acc[k] = fma(lv[k], xr, acc[k]);
            }
            __syncthreads();   // xs consumed
            p = p1;
        }
#pragma unroll
        for (int k = 0; k < TB / 4; ++k)
            for (int o = 16; o; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < TB / 4; ++k) red[half][g + 4 * k] = acc[k];
        }
        __syncthreads();
        if (t < TB) {
            const int i = i0 + t;
            xs[t] = i < n ? tv[i] - (red[0][t] + red[1][t]) : 0.0;
        }
        __syncthreads();
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < TB / 4; ++k) s = fma(dsm[r + TB * (g + 4 * k)], xs[g + 4 * k], s);
        // sum the four column groups: reuse xs beyond the first block as scratch
        xs[TB + g * TB + r] = s;
        __syncthreads();
        if (t < TB && i0 + t < n) {
            x[i0 + t] = xs[TB + t] + xs[2 * TB + t] + xs[3 * TB + t] + xs[4 * TB + t];
            __threadfence();
        }
        __syncthreads();
        if (t == 0) st_release(done, q + 1);
    }
}

}  // namespace

kfb_status TrsvPlan::prepare(const double *L, int n_, cudaStream_t s) {
    n = n_;
    nb = (n + TB - 1) / TB;
    if (n <= 0) return KFB_OK;
    KFB_TRY(dinv.alloc((size_t)nb * TB * TB * sizeof(double), s));
    KFB_TRY(dinvt.alloc((size_t)nb * TB * TB * sizeof(double), s));
    KFB_TRY(sync.alloc(4 * sizeof(int), s));
    KFB_TRY(zero(sync.ptr, 4 * sizeof(int), s));
    trsv_dinv_kernel<<<nb, TB, 0, s>>>(L, n, dinv.as<double>(), dinvt.as<double>());
    KFB_CUDA_TRY(cudaGetLastError());
    int dev = 0, sms = 0, coop = 0, per_sm_l = 0, per_sm_u = 0;
    KFB_CUDA_TRY(cudaGetDevice(&dev));
    KFB_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    KFB_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop)
        return set_error(KFB_ERR_UNSUPPORTED, "the triangular solve needs cooperative launches");
    KFB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_l, trsv_lower_kernel,
                                                               TRSV_THREADS, 0));
    KFB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm_u, trsv_upper_kernel,
                                                               TRSV_THREADS, 0));
    grid = std::min(nb, sms * std::max(1, std::min(per_sm_l, per_sm_u)));
    return KFB_OK;
}

kfb_status TrsvPlan::solve(const double *L, const double *b, double *tmp, double *x,
                           cudaStream_t s) {
    if (n <= 0) return KFB_OK;
    int *done = sync.as<int>(), *err = sync.as<int>() + 2;
    KFB_CUDA_TRY(cudaMemsetAsync(done, 0, 2 * sizeof(int), s));
    const double *dl = dinv.as<double>(), *du = dinvt.as<double>();
    int *done_l = done, *done_u = done + 1;
    void *args_l[] = {(void *)&L, (void *)&n, (void *)&nb, (void *)&dl, (void *)&b,
                      (void *)&tmp, (void *)&done_l, (void *)&err};
    KFB_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)trsv_lower_kernel, dim3(grid),
                                             dim3(TRSV_THREADS), args_l, 0, s));
    const double *tc = tmp;
    void *args_u[] = {(void *)&L, (void *)&n, (void *)&nb, (void *)&du, (void *)&tc,
                      (void *)&x, (void *)&done_u, (void *)&err};
    KFB_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)trsv_upper_kernel, dim3(grid),
                                             dim3(TRSV_THREADS), args_u, 0, s));
    return KFB_OK;
}

kfb_status TrsvPlan::check(cudaStream_t s) {
    if (n <= 0) return KFB_OK;
    int e = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&e, sync.as<int>() + 2, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (e != 0)
        return set_error(KFB_ERR_TIMEOUT, "triangular solve: a block wait gave up");
    return KFB_OK;
}

}  // namespace kfb
