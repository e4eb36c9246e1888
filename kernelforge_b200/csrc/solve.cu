// RFP storage kernels, the RFP Cholesky factorisation / solve (the drop-ins of
// dpftrf / dpftrs and of the FP32 rfp_potrf / rfp_potrs), and the
// mixed-precision KRR and ridge solves.
//
// Every factorisation goes through chol_dense (chol.cu): the RFP array is
// expanded to a dense column-major lower triangle, factored with the panel
// solves and trailing updates on the int8 tensor cores (digit-sliced FP64
// products), and packed back; solves use the blocked FP64 triangular sweeps of
// trsv.cu.  (The reference factors an RFP array in place by LAPACK's
// potrf / trsm / syrk / potrf sequence on its sub-blocks,
// src/curfp_spftrf.cpp:182-292; the dense copy here costs n^2 doubles of HBM,
// which B200 has to spare, and makes every O(n^3) part one tensor-core GEMM.)
#include <cublas_v2.h>

#include <algorithm>
#include <cmath>
#include <functional>
#include <memory>
#include <vector>

#include "chol.h"
#include "kernels_common.cuh"
#include "trsv.h"

namespace kfb {

namespace {

struct Handles {
    cublasHandle_t blas = nullptr;
    int device = -1;
};

kfb_status get_handles(cudaStream_t s, Handles *&out) {
    static thread_local Handles h[16];
    int dev = 0;
    KFB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 16) return set_error(KFB_ERR_UNSUPPORTED, "device index %d", dev);
    Handles &hd = h[dev];
    if (!hd.blas) {
        if (cublasCreate(&hd.blas) != CUBLAS_STATUS_SUCCESS)
            return set_error(KFB_ERR_CUDA, "cublasCreate failed");
        cublasSetMathMode(hd.blas, CUBLAS_PEDANTIC_MATH);  // no reduced-precision shortcuts
    }
    cublasSetStream(hd.blas, s);
    out = &hd;
    return KFB_OK;
}

}  // namespace

// The per-device cuBLAS handle of this thread, bound to stream s (shared with
// the prediction kernels).
kfb_status blas_for_stream(cudaStream_t s, cublasHandle_t *out) {
    Handles *h = nullptr;
    KFB_TRY(get_handles(s, h));
    *out = h->blas;
    return KFB_OK;
}

namespace {

#define KFB_BLAS_TRY(expr)                                                                  \
    do {                                                                                    \
        cublasStatus_t _b = (expr);                                                         \
        if (_b != CUBLAS_STATUS_SUCCESS)                                                    \
            return set_error(KFB_ERR_CUDA, "%s failed: cublas status %d", #expr, (int)_b);  \
    } while (0)

// ------------------------------------------------------------ small kernels
template <class T>
__global__ void add_diag_kernel(T *arf, int n, T l2, int layout) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) arf[sym_index((kfb_layout)layout, n, i, i)] += l2;
}

template <class T>
__global__ void full_to_rfp_kernel(const T *A, int n, int layout, T *arf) {
    const long long i = blockIdx.y * (long long)blockDim.y + threadIdx.y;
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n && j < n && i <= j) arf[sym_index((kfb_layout)layout, n, i, j)] = A[i * n + j];
}

// 32 x 32 tile (rows i0.., columns j0.., i0 >= j0) of an RFP array into
// t[i - i0][j - j0] (FP64), reading along whichever index is contiguous in
// the RFP storage of this tile (both occur: the two triangles of RFP are
// stored transposed to each other).  Block (32, 8).
template <class Tin>
__device__ __forceinline__ void load_rfp_tile(const Tin *__restrict__ arf, int n, int layout,
                                              int i0, int j0, double (*t)[33]) {
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int ib = min(i0 + 1, n - 1), jb = j0;
    const bool along_i = ib > jb && sym_index((kfb_layout)layout, n, ib, jb) ==
                                       sym_index((kfb_layout)layout, n, i0, jb) + 1;
    for (int r = ty; r < 32; r += 8) {
        const int i = along_i ? i0 + tx : i0 + r, j = along_i ? j0 + r : j0 + tx;
        double v = 0.0;
        if (i < n && j < n) v = (double)arf[sym_index((kfb_layout)layout, n, i, j)];
        if (along_i) t[tx][r] = v;
        else t[r][tx] = v;
    }
}

// Full symmetric row-major copy, one lower tile per block writing both
// triangles with coalesced stores.
template <class Tin, class Tout>
__global__ void rfp_to_full_tiled_kernel(const Tin *__restrict__ arf, int n, int layout,
                                         Tout *__restrict__ A) {
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi < bj) return;
    __shared__ double t[32][33];
    const int i0 = bi * 32, j0 = bj * 32;
    load_rfp_tile(arf, n, layout, i0, j0, t);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    for (int r = ty; r < 32; r += 8) {
        const int i = i0 + r, j = j0 + tx;   // A[i][j], along j
        if (i < n && j < n) A[(size_t)i * n + j] = (Tout)t[r][tx];
        const int i2 = j0 + r, j2 = i0 + tx;   // A[j0 + r][i0 + tx] = t[tx][r]
        if (bi != bj && i2 < n && j2 < n) A[(size_t)i2 * n + j2] = (Tout)t[tx][r];
    }
}

// out = sum_i a_i b_i  (FP64), one partial per block then atomically combined
__global__ void dot_kernel(const double *a, const double *b, int n, double *out) {
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        acc = fma(a[i], b[i], acc);
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    __shared__ double part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) atomicAdd(out, v);
    }
}

// y += s * x
__global__ void axpy_kernel(const double *x, double s, int n, double *y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += s * x[i];
}

__global__ void fill_kernel(double *x, double v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = v;
}
// a start vector with no special alignment to the constant vector
__global__ void fill_alt_kernel(double *x, double v, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = (i % 3 == 0 ? -2.0 : 1.0) * v * (1.0 + 1e-3 * (i % 7));
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

// Dense column-major lower triangle of F = B - coef v v^T + diag I, B in RFP
// (FP64 arithmetic, TD result); the upper triangle is not touched.
template <class TD>
__global__ void dense_deflate_kernel(const float *__restrict__ B, int n, int layout,
                                     const double *__restrict__ v, double coef, double diag,
                                     TD *__restrict__ F) {
    // one lower 32 x 32 tile per block; column-major stores along i
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi < bj) return;
    __shared__ double t[32][33];
    const int i0 = bi * 32, j0 = bj * 32;
    load_rfp_tile(B, n, layout, i0, j0, t);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = i0 + tx;
    if (i >= n) return;
    const double vi = v[i];
    for (int r = ty; r < 32; r += 8) {
        const int j = j0 + r;
        if (j >= n || i < j) continue;
        double f = t[tx][r] - coef * vi * v[j];
        if (i == j) f += diag;
        F[(size_t)j * n + i] = (TD)f;
    }
}

// Dense column-major lower FP64 copy of an RFP matrix (FP32 or FP64) with l2
// added to its diagonal; the upper triangle is not touched.  Block (32, 8),
// one lower 32 x 32 tile per block, stores along i.
template <class Tin>
__global__ void rfp_to_dense_lower_kernel(const Tin *__restrict__ B, int n, int layout,
                                          double l2, double *__restrict__ F) {
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi < bj) return;
    __shared__ double t[32][33];
    const int i0 = bi * 32, j0 = bj * 32;
    load_rfp_tile(B, n, layout, i0, j0, t);
    __syncthreads();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int i = i0 + tx;
    if (i >= n) return;
    for (int r = ty; r < 32; r += 8) {
        const int j = j0 + r;
        if (j >= n || i < j) continue;
        F[(size_t)j * n + i] = t[tx][r] + (i == j ? l2 : 0.0);
    }
}

// RFP copy of a dense column-major lower Cholesky factor L: both RFP layouts
// hold L(max(i,j), min(i,j)) at the symmetric position of (i, j) (UPLO='U'
// stores U = L^T).
template <class Tout>
__global__ void dense_lower_to_rfp_kernel(const double *__restrict__ L, int n, int layout,
                                          Tout *__restrict__ arf) {
    const long long i = blockIdx.y * (long long)blockDim.y + threadIdx.y;
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n && j < n && i <= j) arf[sym_index((kfb_layout)layout, n, i, j)] = (Tout)L[i * n + j];
}

__global__ void f32_to_f64_kernel(const float *a, int n, double *b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (double)a[i];
}
__global__ void f64_to_f32_kernel(const double *a, int n, float *b) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) b[i] = (float)a[i];
}


}  // namespace

// ----------------------------------------------------------------- exported
kfb_status rfp_add_diag(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt,
                        cudaStream_t s) {
    if (n <= 0 || l2 == 0.0) return KFB_OK;
    if (dt == KFB_F64)
        add_diag_kernel<double><<<nblk(n, 256), 256, 0, s>>>(static_cast<double *>(arf), n, l2, uplo);
    else
        add_diag_kernel<float><<<nblk(n, 256), 256, 0, s>>>(static_cast<float *>(arf), n, (float)l2, uplo);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

kfb_status full_to_rfp(const void *A, int n, kfb_layout uplo, kfb_dtype dt, void *arf,
                       cudaStream_t s) {
    if (n <= 0) return KFB_OK;
    dim3 blk(32, 8), grd(nblk(n, 32), nblk(n, 8));
    if (dt == KFB_F64)
        full_to_rfp_kernel<double><<<grd, blk, 0, s>>>(static_cast<const double *>(A), n, uplo,
                                                       static_cast<double *>(arf));
    else
        full_to_rfp_kernel<float><<<grd, blk, 0, s>>>(static_cast<const float *>(A), n, uplo,
                                                      static_cast<float *>(arf));
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

kfb_status rfp_to_full(const void *arf, int n, kfb_layout uplo, kfb_dtype dt, void *A,
                       cudaStream_t s) {
    if (n <= 0) return KFB_OK;
    dim3 blk(32, 8), grd(nblk(n, 32), nblk(n, 32));
    if (dt == KFB_F64)
        rfp_to_full_tiled_kernel<double, double><<<grd, blk, 0, s>>>(
            static_cast<const double *>(arf), n, uplo, static_cast<double *>(A));
    else
        rfp_to_full_tiled_kernel<float, float><<<grd, blk, 0, s>>>(
            static_cast<const float *>(arf), n, uplo, static_cast<float *>(A));
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

// Digit planes of the tensor-core Cholesky updates for a factor held in dt:
// 7 (FP64-class) for an FP64 matrix, 4 (about 27 significant bits, FP32-class)
// for an FP32 one.
inline int chol_slices(kfb_dtype dt) { return dt == KFB_F64 ? 7 : 4; }

// Dense column-major lower FP64 copy of an RFP array plus l2 on the diagonal.
kfb_status rfp_to_dense_lower(const void *arf, int n, kfb_layout uplo, kfb_dtype dt, double l2,
                              double *F, cudaStream_t s) {
    const dim3 b2(32, 8), gt(nblk(n, 32), nblk(n, 32));
    if (dt == KFB_F64)
        rfp_to_dense_lower_kernel<double><<<gt, b2, 0, s>>>(static_cast<const double *>(arf), n,
                                                            uplo, l2, F);
    else
        rfp_to_dense_lower_kernel<float><<<gt, b2, 0, s>>>(static_cast<const float *>(arf), n,
                                                           uplo, l2, F);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

kfb_status dense_lower_to_rfp(const double *L, int n, kfb_layout uplo, kfb_dtype dt, void *arf,
                              cudaStream_t s) {
    const dim3 b2(32, 8), g2(nblk(n, 32), nblk(n, 8));
    if (dt == KFB_F64)
        dense_lower_to_rfp_kernel<double><<<g2, b2, 0, s>>>(L, n, uplo, static_cast<double *>(arf));
    else
        dense_lower_to_rfp_kernel<float><<<g2, b2, 0, s>>>(L, n, uplo, static_cast<float *>(arf));
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

// In-place RFP Cholesky of (A + l2 I): the RFP array is expanded to a dense
// column-major FP64 lower triangle, factored by chol_dense (tensor-core panel
// solves and trailing updates) and packed back into the same RFP layout and
// element type.  On a non-positive pivot *info is set and arf is unchanged.
kfb_status rfp_potrf(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt, int *info,
                     cudaStream_t s) {
    *info = 0;
    if (n <= 0) return KFB_OK;
    TraceScope tr("rfp_potrf", s);
    DevBuf F;
    KFB_TRY(F.alloc((size_t)n * n * sizeof(double), s));
    KFB_TRY(rfp_to_dense_lower(arf, n, uplo, dt, l2, F.as<double>(), s));
    KFB_TRY(chol_dense(F.as<double>(), n, n, chol_slices(dt), info, s));
    if (*info != 0) return KFB_OK;
    return dense_lower_to_rfp(F.as<double>(), n, uplo, dt, arf, s);
}

// Solve with an RFP factor: the factor is expanded to a dense FP64 lower
// triangle and each right-hand side goes through the two blocked triangular
// sweeps of trsv.cu (in FP64; FP32 right-hand sides are widened and narrowed).
kfb_status rfp_potrs(const void *arf, void *B, int n, int nrhs, kfb_layout uplo, kfb_dtype dt,
                     cudaStream_t s) {
    if (n <= 0 || nrhs <= 0) return KFB_OK;
    TraceScope tr("rfp_potrs", s);
    DevBuf F, x, tmp;
    KFB_TRY(F.alloc((size_t)n * n * sizeof(double), s));
    KFB_TRY(rfp_to_dense_lower(arf, n, uplo, dt, 0.0, F.as<double>(), s));
    TrsvPlan plan;
    KFB_TRY(plan.prepare(F.as<double>(), n, s));
    KFB_TRY(tmp.alloc((size_t)n * sizeof(double), s));
    if (dt == KFB_F32) KFB_TRY(x.alloc((size_t)n * sizeof(double), s));
    for (int c = 0; c < nrhs; ++c) {
        if (dt == KFB_F64) {
            double *b = static_cast<double *>(B) + (size_t)c * n;
            KFB_TRY(plan.solve(F.as<double>(), b, tmp.as<double>(), b, s));
        } else {
            float *b = static_cast<float *>(B) + (size_t)c * n;
            f32_to_f64_kernel<<<nblk(n, 256), 256, 0, s>>>(b, n, x.as<double>());
            KFB_TRY(plan.solve(F.as<double>(), x.as<double>(), tmp.as<double>(), x.as<double>(), s));
            f64_to_f32_kernel<<<nblk(n, 256), 256, 0, s>>>(x.as<double>(), n, b);
            KFB_CUDA_TRY(cudaGetLastError());
        }
    }
    return plan.check(s);
}

namespace {

// (A + lam I) x of the operator a mixed solve refines against, FP64 vectors
using ApplyFn = std::function<kfb_status(const double *x, double lam, double *out)>;

// out = (K + l2 I) x with K dense FP32 or FP64 (row-major, symmetric), one
// warp per row, FP64 accumulation
template <class TK>
__global__ void dense_apply_kernel(const TK *__restrict__ K, const double *__restrict__ x,
                                   int n, double l2, double *__restrict__ out) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    const TK *kr = K + (size_t)row * n;
    double acc = 0.0;
    for (int j = lane; j < n; j += 32) acc = fma((double)kr[j], x[j], acc);
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) out[row] = acc + l2 * x[row];
}

// t[m] = sum_c z[m][c] x[c] (FP32 features, FP64 accumulation), one warp per row
__global__ void zx_kernel(const float *__restrict__ z, const double *__restrict__ x, int nm,
                          int d, double *__restrict__ t) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= nm) return;
    const float *zr = z + (size_t)row * d;
    double acc = 0.0;
    for (int c = lane; c < d; c += 32) acc = fma((double)zr[c], x[c], acc);
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) t[row] = acc;
}

// zty[c] += sum_m z[m][c] y[m] (FP64 accumulation), one thread per column,
// molecules split over blockIdx.y and combined with atomics
__global__ void zty_kernel(const float *__restrict__ z, const double *__restrict__ y, int nm,
                           int d, int mchunk, double *__restrict__ zty) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= d) return;
    const int m0 = blockIdx.y * mchunk, m1 = min(nm, m0 + mchunk);
    double t = 0.0;
    for (int m = m0; m < m1; ++m) t += (double)z[(size_t)m * d + c] * y[m];
    atomicAdd(zty + c, t);
}

// z1[m][c] = z[m][c] - t[m] v[c] with t = z v: the features with the dominant
// direction v of Z^T Z projected out (FP64 arithmetic, FP32 result)
__global__ void project_out_kernel(const float *__restrict__ z, const double *__restrict__ t,
                                   const double *__restrict__ v, long long nm, int d,
                                   float *__restrict__ z1) {
    const long long n = nm * d;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const long long m = i / d;
        const int c = (int)(i - m * d);
        z1[i] = (float)((double)z[i] - t[m] * v[c]);
    }
}

// ---- device-resident scalars of the iterative solves: the dot products,
// step lengths and norms stay on the device, so an iteration enqueues its
// kernels without waiting for the host; the host reads a pair (rr, flag)
// once per CG iteration, one iteration behind, to stop.
enum : int {
    S_NRM = 0, S_VAV, S_WAW, S_WW, S_VW, S_LAM2, S_PQ, S_RZ0, S_RZ1, S_WR, S_Y2,
    S_RR, S_FLAG,  // adjacent: copied to the host together
    S_COUNT = 16
};

// out[slot] = 0 for the listed slots
__global__ void zero_slots_kernel(double *sc, int a, int b, int c) {
    if (threadIdx.x == 0) {
        if (a >= 0) sc[a] = 0.0;
        if (b >= 0) sc[b] = 0.0;
        if (c >= 0) sc[c] = 0.0;
    }
}
// out = a / sqrt(sc[i]) (a unchanged if sc[i] <= 0)
__global__ void scale_rsqrt_kernel(const double *a, const double *sc, int i, int n, double *out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const double t = sc[i];
    if (k < n) out[k] = t > 0.0 ? a[k] / sqrt(t) : a[k];
}
// y += mult * sc[i] * x
__global__ void axpy_dev_kernel(const double *x, const double *sc, int i, double mult, int n,
                                double *y) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) y[k] += mult * sc[i] * x[k];
}
// sc[LAM2] = max(sc[LAM2], sc[WAW] / sc[WW])
__global__ void lam2_update_kernel(double *sc) {
    if (threadIdx.x == 0) {
        const double ww = sc[S_WW];
        if (ww > 0.0) sc[S_LAM2] = fmax(sc[S_LAM2], sc[S_WAW] / ww);
    }
}
// CG update with alpha = rz / pq from the device: x += alpha p, r -= alpha q.
// A non-positive curvature with a nonzero residual raises the flag.
__global__ void cg_update_kernel(const double *p, const double *q, double *x, double *r, int n,
                                 double *sc, int rz_slot) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const double pq = sc[S_PQ], rz = sc[rz_slot];
    const double a = pq > 0.0 ? rz / pq : 0.0;
    if (k == 0 && !(pq > 0.0) && rz > 0.0) sc[S_FLAG] = 1.0;
    if (k < n) {
        x[k] += a * p[k];
        r[k] -= a * q[k];
    }
}
// p = z + beta p with beta = sc[new] / sc[old]
__global__ void xpby_dev_kernel(const double *z, const double *sc, int new_slot, int old_slot,
                                int n, double *p) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const double o = sc[old_slot];
    const double beta = o > 0.0 ? sc[new_slot] / o : 0.0;
    if (k < n) p[k] = z[k] + beta * p[k];
}

struct DevScalars {
    DevBuf buf;
    double *host = nullptr;  // pinned, 4 doubles: two (rr, flag) pairs
    cudaEvent_t ev[2] = {nullptr, nullptr};
    kfb_status init(cudaStream_t s) {
        KFB_TRY(buf.alloc(S_COUNT * sizeof(double), s));
        KFB_TRY(zero(buf.ptr, S_COUNT * sizeof(double), s));
        // pinned host slots, allocated once per thread (cudaMallocHost synchronises)
        static thread_local double *pinned = nullptr;
        if (!pinned) KFB_CUDA_TRY(cudaMallocHost(&pinned, 4 * sizeof(double)));
        host = pinned;
        for (auto &e : ev) KFB_CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        return KFB_OK;
    }
    ~DevScalars() {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    }
    double *sc() const { return buf.as<double>(); }
    // sc[slot] += a . b (the slot is zeroed first), no host wait
    kfb_status dot(const double *a, const double *b, int n, int slot, cudaStream_t s) {
        zero_slots_kernel<<<1, 32, 0, s>>>(sc(), slot, -1, -1);
        dot_kernel<<<std::min(nblk(n, 256), 1184u), 256, 0, s>>>(a, b, n, sc() + slot);
        KFB_CUDA_TRY(cudaGetLastError());
        return KFB_OK;
    }
    kfb_status read(int slot, double &out, cudaStream_t s) {
        KFB_CUDA_TRY(cudaMemcpyAsync(&out, sc() + slot, sizeof(double), cudaMemcpyDeviceToHost, s));
        KFB_CUDA_TRY(cudaStreamSynchronize(s));
        return KFB_OK;
    }
};

// The dominant eigenpair (mu, v) of a symmetric positive semi-definite
// operator by 20 power steps, and lam2, an upper estimate of the norm of the
// operator with that pair removed (8 power steps orthogonal to v; Rayleigh
// quotients approach the norm from below, hence the factor 1.5).  All on the
// device; one host read at the end.
kfb_status power_dominant(const ApplyFn &A, int n, double *v, double *w, double *tmp,
                          DevScalars &ds, cudaStream_t s, double &mu, double &lam2) {
    const unsigned gb = nblk(n, 256);
    double *sc = ds.sc();
    fill_kernel<<<gb, 256, 0, s>>>(v, 1.0 / std::sqrt((double)n), n);
    for (int k = 0; k < 20; ++k) {
        KFB_TRY(A(v, 0.0, tmp));
        KFB_TRY(ds.dot(v, tmp, n, S_VAV, s));
        KFB_TRY(ds.dot(tmp, tmp, n, S_NRM, s));
        scale_rsqrt_kernel<<<gb, 256, 0, s>>>(tmp, sc, S_NRM, n, v);
    }
    zero_slots_kernel<<<1, 32, 0, s>>>(sc, S_LAM2, -1, -1);
    fill_alt_kernel<<<gb, 256, 0, s>>>(w, 1.0 / std::sqrt((double)n), n);
    for (int k = 0; k < 8; ++k) {
        KFB_TRY(ds.dot(v, w, n, S_VW, s));
        axpy_dev_kernel<<<gb, 256, 0, s>>>(v, sc, S_VW, -1.0, n, w);
        KFB_TRY(A(w, 0.0, tmp));
        KFB_TRY(ds.dot(w, tmp, n, S_WAW, s));
        KFB_TRY(ds.dot(w, w, n, S_WW, s));
        KFB_TRY(ds.dot(tmp, tmp, n, S_NRM, s));
        lam2_update_kernel<<<1, 32, 0, s>>>(sc);
        scale_rsqrt_kernel<<<gb, 256, 0, s>>>(tmp, sc, S_NRM, n, w);
    }
    KFB_CUDA_TRY(cudaGetLastError());
    double h[S_COUNT];
    KFB_CUDA_TRY(cudaMemcpyAsync(h, sc, sizeof(h), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    mu = h[S_VAV];
    lam2 = 1.5 * h[S_LAM2];
    return KFB_OK;
}

// Mixed-precision solve of (A + l2 I) x = y.  The FP32 factor is of
//   F = B - fcoef v v^T + (lam + shift) I       (B an FP32 RFP matrix)
// chosen so that F + defl v v^T approximates A + lam I; the preconditioner
//   M^{-1} = (F + defl v v^T)^{-1}
// is applied with the Sherman-Morrison formula, and conjugate gradients in
// FP64 refine against the operator A itself.  With the dominant eigenvalue mu
// of A removed from the factor (defl = mu - lam2) its eigenvalue along v is
// about lam2 rather than ~0, so F^{-1} v stays bounded and the Sherman-Morrison
// correction does not cancel.  The shift starts at max(0, 2 u32 lam2 - lam)
// and grows 4x per failed factorisation; CG meeting a non-positive curvature
// p^T (A + lam I) p means A + lam I is indefinite at the precision A is held
// in (KFB_ERR_NOT_PD; with KFB_SOLVE_LAMBDA_FLOOR lam is raised x10 instead).
kfb_status mixed_core(const ApplyFn &A, const float *B, int n, kfb_layout uplo, const double *v,
                      double fcoef, double defl, double lam2, const double *y, double l2,
                      double tol, int maxit, int flags, double *alpha, kfb_solve_info &inf,
                      DevScalars &ds, cudaStream_t s) {
    DevBuf r, z, p, q, dw;
    KFB_TRY(r.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(z.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(p.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(q.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(dw.alloc((size_t)n * sizeof(double), s));
    const unsigned gb = nblk(n, 256);
    const double u32 = 5.960464477539063e-08;
    double *sc = ds.sc();
    KFB_TRY(ds.dot(y, y, n, S_Y2, s));
    double ynorm2 = 0.0;
    KFB_TRY(ds.read(S_Y2, ynorm2, s));
    const double ynorm = std::sqrt(ynorm2);
    KFB_TRY(zero(alpha, (size_t)n * sizeof(double), s));
    if (ynorm == 0.0) return KFB_OK;

    // The factor: the dense lower triangle of F factored by chol_dense (panel
    // solves and trailing updates on the int8 tensor cores) with 4 digit planes
    // (FP32-class: the precision asked of the preconditioner) or, with
    // KFB_SOLVE_FP64_FACTOR, 6 (42-bit digits: as a preconditioner of the FP64
    // conjugate gradients it needs as few steps as 7 planes, two at n = 10,000,
    // for 21 instead of 28 int8 products per update); held in FP64 either way,
    // so the preconditioner out = F^{-1} x is the pair of blocked FP64 sweeps
    // of trsv.cu.
    const bool f64 = (flags & KFB_SOLVE_FP64_FACTOR) != 0;
    DevBuf Fd, ttmp;
    TrsvPlan trsv;
    KFB_TRY(Fd.alloc((size_t)n * n * sizeof(double), s));
    KFB_TRY(ttmp.alloc((size_t)n * sizeof(double), s));
    auto factor = [&](double diag, int &finfo) -> kfb_status {
        const dim3 b2(32, 8), gt(nblk(n, 32), nblk(n, 32));
        dense_deflate_kernel<double><<<gt, b2, 0, s>>>(B, n, uplo, v, fcoef, diag,
                                                       Fd.as<double>());
        KFB_CUDA_TRY(cudaGetLastError());
        KFB_TRY(chol_dense(Fd.as<double>(), n, n, f64 ? 6 : 4, &finfo, s));
        if (finfo == 0) KFB_TRY(trsv.prepare(Fd.as<double>(), n, s));
        return KFB_OK;
    };
    auto solve_f_dev = [&](const double *x, int slot, double *out) -> kfb_status {
        (void)slot;
        TraceScope tr_s("mixed:potrs", s);
        return trsv.solve(Fd.as<double>(), x, ttmp.as<double>(), out, s);
    };

    auto attempt = [&](double lam) -> kfb_status {
        double shift = std::max(0.0, 2.0 * u32 * lam2 - lam);
        int finfo = 0;
        auto tr_f = std::make_unique<TraceScope>("mixed:factor", s);
        for (int a = 0; a < 12; ++a) {
            KFB_TRY(factor(lam + shift, finfo));
            if (finfo == 0) break;
            // an FP64 factor that fails means A + lam I itself is indefinite at
            // the precision A is held in: under the lambda floor, raise lam
            // rather than shift a preconditioner for an indefinite system
            if (f64 && (flags & KFB_SOLVE_LAMBDA_FLOOR)) break;
            shift = (shift == 0.0) ? std::max(u32 * lam2, 10.0 * lam) : shift * 4.0;
        }
        inf.factor_info = finfo;
        inf.shift = shift;
        if (finfo != 0)
            return set_error(KFB_ERR_NOT_PD,
                             "the preconditioner's Cholesky failed even with shift %g (info=%d)",
                             shift, finfo);
        tr_f.reset();
        TraceScope tr_cg("mixed:cg", s);
        // w = F^{-1} v (v has unit norm: slot S_NRM set to 1 for the scaling);
        // without deflation (defl = 0) there is no correction to apply
        double sm_coef = 0.0;
        if (defl != 0.0) {
            const double one = 1.0;
            KFB_CUDA_TRY(cudaMemcpyAsync(sc + S_NRM, &one, sizeof(double), cudaMemcpyHostToDevice,
                                         s));
            KFB_TRY(solve_f_dev(v, S_NRM, dw.as<double>()));
            double vfv = 0.0;
            KFB_TRY(ds.dot(v, dw.as<double>(), n, S_VW, s));
            KFB_TRY(ds.read(S_VW, vfv, s));
            sm_coef = defl / (1.0 + defl * vfv);
        }
        // M^{-1} x = F^{-1} x - sm_coef (w . x) w, with |x|^2 in sc[slot]
        auto precond = [&](const double *x, int slot, double *out) -> kfb_status {
            KFB_TRY(solve_f_dev(x, slot, out));
            if (sm_coef == 0.0) return KFB_OK;
            KFB_TRY(ds.dot(dw.as<double>(), x, n, S_WR, s));
            axpy_dev_kernel<<<gb, 256, 0, s>>>(dw.as<double>(), sc, S_WR, -sm_coef, n, out);
            KFB_CUDA_TRY(cudaGetLastError());
            return KFB_OK;
        };
        // preconditioned conjugate gradients in FP64 from alpha = 0; when the
        // recurrence residual meets the tolerance but the true one y - A alpha
        // does not (their gap grows with the condition number), CG restarts
        // from alpha with the true residual (at most 4 restarts)
        KFB_TRY(zero(alpha, (size_t)n * sizeof(double), s));
        int total_it = 0;
        double rel = 0.0;
        for (int restart = 0; restart < 5; ++restart) {
            // r = y - (A + lam I) alpha
            KFB_CUDA_TRY(cudaMemcpyAsync(r.ptr, y, (size_t)n * sizeof(double),
                                         cudaMemcpyDeviceToDevice, s));
            if (restart > 0) {
                KFB_TRY(A(alpha, lam, q.as<double>()));
                axpy_kernel<<<gb, 256, 0, s>>>(q.as<double>(), -1.0, n, r.as<double>());
            }
            zero_slots_kernel<<<1, 32, 0, s>>>(sc, S_FLAG, -1, -1);
            KFB_TRY(ds.dot(r.as<double>(), r.as<double>(), n, S_RR, s));
            KFB_TRY(precond(r.as<double>(), S_RR, z.as<double>()));
            KFB_CUDA_TRY(cudaMemcpyAsync(p.ptr, z.ptr, (size_t)n * sizeof(double),
                                         cudaMemcpyDeviceToDevice, s));
            KFB_TRY(ds.dot(r.as<double>(), z.as<double>(), n, S_RZ0, s));
            int it = 0;
            bool indefinite = false;
            const int budget = maxit - total_it;
            for (; it < budget; ++it) {
                const int rz_cur = (it & 1) ? S_RZ1 : S_RZ0, rz_new = (it & 1) ? S_RZ0 : S_RZ1;
                KFB_TRY(A(p.as<double>(), lam, q.as<double>()));  // q = (A + lam I) p
                KFB_TRY(ds.dot(p.as<double>(), q.as<double>(), n, S_PQ, s));
                cg_update_kernel<<<gb, 256, 0, s>>>(p.as<double>(), q.as<double>(), alpha,
                                                    r.as<double>(), n, sc, rz_cur);
                KFB_TRY(ds.dot(r.as<double>(), r.as<double>(), n, S_RR, s));
                KFB_CUDA_TRY(cudaMemcpyAsync(ds.host + 2 * (it & 1), sc + S_RR,
                                             2 * sizeof(double), cudaMemcpyDeviceToHost, s));
                KFB_CUDA_TRY(cudaEventRecord(ds.ev[it & 1], s));
                if (f64) {
                    // an FP64 factor converges in one or two steps: test this
                    // step's residual before paying for another preconditioner
                    // solve (the FP32 path instead tests one step behind)
                    KFB_CUDA_TRY(cudaEventSynchronize(ds.ev[it & 1]));
                    const double rr = ds.host[2 * (it & 1)], fl = ds.host[2 * (it & 1) + 1];
                    if (fl != 0.0) {
                        indefinite = true;
                        break;
                    }
                    if (std::sqrt(rr) <= tol * ynorm) {
                        ++it;
                        break;
                    }
                }
                KFB_TRY(precond(r.as<double>(), S_RR, z.as<double>()));
                KFB_TRY(ds.dot(r.as<double>(), z.as<double>(), n, rz_new, s));
                xpby_dev_kernel<<<gb, 256, 0, s>>>(z.as<double>(), sc, rz_new, rz_cur, n,
                                                   p.as<double>());
                KFB_CUDA_TRY(cudaGetLastError());
                // stop test on the previous iteration's residual (the device runs one ahead)
                const int chk = it - 1;
                if (!f64 && chk >= 0) {
                    KFB_CUDA_TRY(cudaEventSynchronize(ds.ev[chk & 1]));
                    const double rr = ds.host[2 * (chk & 1)], fl = ds.host[2 * (chk & 1) + 1];
                    if (fl != 0.0) {
                        indefinite = true;
                        it = chk;
                        break;
                    }
                    if (std::sqrt(rr) <= tol * ynorm) {
                        ++it;
                        break;
                    }
                }
            }
            if (!indefinite && it > 0 && it >= budget) {
                KFB_CUDA_TRY(cudaEventSynchronize(ds.ev[(it - 1) & 1]));
                if (ds.host[2 * ((it - 1) & 1) + 1] != 0.0) indefinite = true;
            }
            total_it += it;
            if (indefinite) {
                KFB_TRY(trsv.check(s));
                inf.iterations = total_it;
                return set_error(KFB_ERR_NOT_PD,
                                 "the system is indefinite at the precision of its matrix "
                                 "(non-positive p^T A p after %d CG iterations, l2 = %g); use a "
                                 "larger l2",
                                 total_it, lam);
            }
            // true residual of alpha
            KFB_TRY(A(alpha, lam, q.as<double>()));
            KFB_CUDA_TRY(cudaMemcpyAsync(r.ptr, y, (size_t)n * sizeof(double),
                                         cudaMemcpyDeviceToDevice, s));
            axpy_kernel<<<gb, 256, 0, s>>>(q.as<double>(), -1.0, n, r.as<double>());
            KFB_TRY(ds.dot(r.as<double>(), r.as<double>(), n, S_RR, s));
            double rr = 0.0;
            KFB_TRY(ds.read(S_RR, rr, s));
            rel = std::sqrt(rr) / ynorm;
            if (rel <= tol || total_it >= maxit) break;
        }
        KFB_TRY(trsv.check(s));
        inf.iterations = total_it;
        inf.used_cg = 1;
        inf.rel_residual = rel;
        if (inf.rel_residual > tol)
            return set_error(KFB_ERR_NO_CONVERGENCE,
                             "refinement stopped at relative residual %.3e (tol %.1e) after %d "
                             "iterations",
                             inf.rel_residual, tol, total_it);
        return KFB_OK;
    };

    double lam = l2;
    kfb_status st = KFB_OK;
    for (int tries = 0; tries < 10; ++tries) {
        st = attempt(lam);
        inf.lambda_eff = lam;
        if (st != KFB_ERR_NOT_PD || !(flags & KFB_SOLVE_LAMBDA_FLOOR)) break;
        // raise the regularisation until A + lam I is definite at FP32 precision;
        // the first step goes to u32 lam2 (the FP64-factor path skipped the
        // power steps, so it estimates lam2 now, with p, q, z as scratch)
        if (tries == 0 && lam2 == 0.0) {
            double mu_e = 0.0;
            KFB_TRY(power_dominant(A, n, p.as<double>(), q.as<double>(), z.as<double>(), ds, s,
                                   mu_e, lam2));
        }
        lam = (tries == 0) ? std::max(10.0 * l2, u32 * lam2) : lam * 10.0;
    }
    return st;
}

}  // namespace

namespace {
// r = y - r
__global__ void rsub_kernel(const double *y, int n, double *r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = y[i] - r[i];
}
}  // namespace

// FP64 kernel ridge solve behind kernelmath.cho_solve_rfp: the FP64-class
// tensor-core Cholesky (7 digit planes) of K + l2 I, the two blocked triangular
// sweeps, and two steps of iterative refinement against K itself (residual
// y - (K + l2 I) alpha from a dense FP64 copy of K), which bring alpha to the
// accuracy of an FP64 LAPACK solve; the factor is then written over the RFP
// input in its layout, as dpftrf does (src/math.cpp:134-171).
kfb_status cho_solve_rfp_f64(double *arf, const double *y, int n, double l2, kfb_layout uplo,
                             double *alpha, int *info, cudaStream_t s) {
    *info = 0;
    if (n <= 0) return KFB_OK;
    TraceScope tr("cho_solve_rfp", s);
    DevBuf D, F, r, tmp;
    KFB_TRY(D.alloc((size_t)n * n * sizeof(double), s));
    KFB_TRY(F.alloc((size_t)n * n * sizeof(double), s));
    KFB_TRY(r.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(tmp.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(rfp_to_full(arf, n, uplo, KFB_F64, D.ptr, s));
    KFB_TRY(rfp_to_dense_lower(arf, n, uplo, KFB_F64, l2, F.as<double>(), s));
    KFB_TRY(chol_dense(F.as<double>(), n, n, 7, info, s));
    if (*info != 0) return KFB_OK;
    TrsvPlan plan;
    KFB_TRY(plan.prepare(F.as<double>(), n, s));
    KFB_TRY(plan.solve(F.as<double>(), y, tmp.as<double>(), alpha, s));
    const unsigned gw = nblk((long long)n * 32, 256), gb = nblk(n, 256);
    for (int it = 0; it < 2; ++it) {
        dense_apply_kernel<double><<<gw, 256, 0, s>>>(D.as<double>(), alpha, n, l2, r.as<double>());
        rsub_kernel<<<gb, 256, 0, s>>>(y, n, r.as<double>());
        KFB_CUDA_TRY(cudaGetLastError());
        KFB_TRY(plan.solve(F.as<double>(), r.as<double>(), tmp.as<double>(), r.as<double>(), s));
        axpy_kernel<<<gb, 256, 0, s>>>(r.as<double>(), 1.0, n, alpha);
        KFB_CUDA_TRY(cudaGetLastError());
    }
    KFB_TRY(plan.check(s));
    return dense_lower_to_rfp(F.as<double>(), n, uplo, KFB_F64, arf, s);
}

// Kernel ridge: A = K (FP32 RFP input, expanded to a dense FP32 copy for the
// FP64 residual products); the factor deflates K's dominant eigenpair.
kfb_status krr_solve_mixed(const float *k_rfp, const double *y, int n, double l2,
                           kfb_layout uplo, double tol, int maxit, int flags, double *alpha,
                           kfb_solve_info *info, cudaStream_t s) {
    kfb_solve_info inf{};
    inf.lambda_eff = l2;
    DevBuf Kd, dv, dw, dtmp;
    TraceScope tr_all("krr_solve", s);
    KFB_TRY(Kd.alloc((size_t)n * n * sizeof(float), s));
    KFB_TRY(rfp_to_full(k_rfp, n, uplo, KFB_F32, Kd.ptr, s));
    KFB_TRY(dv.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(dw.alloc((size_t)n * sizeof(double), s));
    KFB_TRY(dtmp.alloc((size_t)n * sizeof(double), s));
    DevScalars ds;
    KFB_TRY(ds.init(s));
    const unsigned gw = nblk((long long)n * 32, 256);
    ApplyFn A = [&](const double *x, double lam, double *out) -> kfb_status {
        TraceScope tr_a("mixed:apply", s);
        dense_apply_kernel<float><<<gw, 256, 0, s>>>(Kd.as<float>(), x, n, lam, out);
        KFB_CUDA_TRY(cudaGetLastError());
        return KFB_OK;
    };
    double ynorm2 = 0.0;
    KFB_TRY(ds.dot(y, y, n, S_Y2, s));
    KFB_TRY(ds.read(S_Y2, ynorm2, s));
    if (ynorm2 == 0.0) {
        KFB_TRY(zero(alpha, (size_t)n * sizeof(double), s));
        if (info) *info = inf;
        return KFB_OK;
    }
    double mu = 0.0, lam2 = 0.0;
    if (flags & KFB_SOLVE_FP64_FACTOR) {
        // an FP64 factor needs no deflation: its rounding (~1e-16 |K|) is far
        // below any usable lambda
        KFB_TRY(zero(dv.ptr, (size_t)n * sizeof(double), s));
    } else {
        TraceScope tr("krr_solve:power", s);
        KFB_TRY(power_dominant(A, n, dv.as<double>(), dw.as<double>(), dtmp.as<double>(), ds, s,
                               mu, lam2));
    }
    const double defl = std::max(0.0, mu - lam2);
    TraceScope tr_core("krr_solve:factor+cg", s);
    const kfb_status st = mixed_core(A, k_rfp, n, uplo, dv.as<double>(), defl, defl, lam2, y, l2,
                                     tol, maxit, flags, alpha, inf, ds, s);
    if (info) *info = inf;
    return st;
}

// Linear ridge on features: (Z^T Z + l2 I) w = Z^T y with Z (nm, d) FP32.  The
// operator is applied matrix-free from Z (two FP64-accumulated passes), so the
// refinement converges to the solution of the exact normal equations, not of
// their FP32 rounding.  The FP32 factor is built from Z with the dominant
// direction v projected out before the SYRK: Z^T Z's entries are dominated by
// its top eigenvalue (the mode shared by all molecules), and forming Z1^T Z1
// with Z1 = Z (I - v v^T) keeps the FP32 rounding at the scale of the
// remaining spectrum.
kfb_status ridge_solve_mixed(const float *zf, const double *y, int nm, int d, double l2,
                             double tol, int maxit, int flags, double *w, kfb_solve_info *info,
                             cudaStream_t s) {
    kfb_solve_info inf{};
    inf.lambda_eff = l2;
    Handles *hd = nullptr;
    KFB_TRY(get_handles(s, hd));
    DevBuf t, rhs, dv, dw, dtmp;
    KFB_TRY(t.alloc((size_t)nm * sizeof(double), s));
    KFB_TRY(rhs.alloc((size_t)d * sizeof(double), s));
    KFB_TRY(dv.alloc((size_t)d * sizeof(double), s));
    KFB_TRY(dw.alloc((size_t)d * sizeof(double), s));
    KFB_TRY(dtmp.alloc((size_t)d * sizeof(double), s));
    DevScalars ds;
    KFB_TRY(ds.init(s));
    const int mchunk = 256;
    const dim3 gty(nblk(d, 128), nblk(nm, mchunk));
    const unsigned gzx = nblk((long long)nm * 32, 256);
    ApplyFn A = [&](const double *x, double lam, double *out) -> kfb_status {
        zx_kernel<<<gzx, 256, 0, s>>>(zf, x, nm, d, t.as<double>());
        KFB_CUDA_TRY(cudaGetLastError());
        KFB_TRY(zero(out, (size_t)d * sizeof(double), s));
        zty_kernel<<<gty, 128, 0, s>>>(zf, t.as<double>(), nm, d, mchunk, out);
        KFB_CUDA_TRY(cudaGetLastError());
        if (lam != 0.0) axpy_kernel<<<nblk(d, 256), 256, 0, s>>>(x, lam, d, out);
        KFB_CUDA_TRY(cudaGetLastError());
        return KFB_OK;
    };
    KFB_TRY(zero(rhs.ptr, (size_t)d * sizeof(double), s));
    zty_kernel<<<gty, 128, 0, s>>>(zf, y, nm, d, mchunk, rhs.as<double>());
    KFB_CUDA_TRY(cudaGetLastError());
    double mu = 0.0, lam2 = 0.0;
    KFB_TRY(power_dominant(A, d, dv.as<double>(), dw.as<double>(), dtmp.as<double>(), ds, s, mu,
                           lam2));
    // B = Z1^T Z1 in RFP, Z1 = Z with v projected out
    DevBuf z1, full, B;
    KFB_TRY(z1.alloc((size_t)nm * d * sizeof(float), s));
    zx_kernel<<<gzx, 256, 0, s>>>(zf, dv.as<double>(), nm, d, t.as<double>());
    project_out_kernel<<<std::min<unsigned>(nblk((long long)nm * d, 256), 148u * 32), 256, 0, s>>>(
        zf, t.as<double>(), dv.as<double>(), nm, d, z1.as<float>());
    KFB_CUDA_TRY(cudaGetLastError());
    KFB_TRY(full.alloc((size_t)d * d * sizeof(float), s));
    const float one = 1.f, zero_f = 0.f;
    KFB_BLAS_TRY(cublasSsyrk(hd->blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, d, nm, &one,
                             z1.as<float>(), d, &zero_f, full.as<float>(), d));
    z1.release();
    KFB_TRY(B.alloc((size_t)d * (d + 1) / 2 * sizeof(float), s));
    KFB_TRY(full_to_rfp(full.ptr, d, KFB_RFP_L, KFB_F32, B.ptr, s));
    full.release();
    const double defl = std::max(0.0, mu - lam2);
    // F = B + lam2 v v^T (eigenvalue ~lam2 along v), M = F + defl v v^T ~ Z^T Z
    const kfb_status st = mixed_core(A, B.as<float>(), d, KFB_RFP_L, dv.as<double>(), -lam2, defl,
                                     lam2, rhs.as<double>(), l2, tol, maxit, flags, w, inf, ds,
                                     s);
    if (info) *info = inf;
    return st;
}

// ---------------------------------------------------------------- normal equations
namespace {

// mirror the upper triangle (row-major) of a symmetric d x d array into its lower
__global__ void mirror_upper_kernel(float *a, int d) {
    const long long i = blockIdx.y * (long long)blockDim.y + threadIdx.y;
    const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < d && j < d && i > j) a[i * d + j] = a[j * d + i];
}

}  // namespace

kfb_status feature_gramian(const float *z, const double *y, int nm, int d, kfb_layout layout,
                           float *ztz, double *zty, cudaStream_t s) {
    Handles *hd = nullptr;
    KFB_TRY(get_handles(s, hd));
    // Z is (nm, d) row-major = a column-major d x nm matrix Zc; Z^T Z = Zc Zc^T.
    // SYRK fills the column-major lower triangle = the row-major upper one.
    DevBuf full;
    float *dense = ztz;
    if (layout != KFB_DENSE) {
        KFB_TRY(full.alloc((size_t)d * d * sizeof(float), s));
        dense = full.as<float>();
    }
    const float one = 1.f, zero_f = 0.f;
    KFB_BLAS_TRY(cublasSsyrk(hd->blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, d, nm, &one, z, d,
                             &zero_f, dense, d));
    dim3 blk(32, 8), grd(nblk(d, 32), nblk(d, 8));
    if (layout == KFB_DENSE) {
        mirror_upper_kernel<<<grd, blk, 0, s>>>(dense, d);
        KFB_CUDA_TRY(cudaGetLastError());
    } else {
        KFB_TRY(full_to_rfp(dense, d, layout, KFB_F32, ztz, s));
    }
    if (y && zty) {
        KFB_TRY(zero(zty, (size_t)d * sizeof(double), s));
        const int mchunk = 256;
        zty_kernel<<<dim3(nblk(d, 128), nblk(nm, mchunk)), 128, 0, s>>>(z, y, nm, d, mchunk, zty);
        KFB_CUDA_TRY(cudaGetLastError());
    }
    return KFB_OK;
}

}  // namespace kfb
