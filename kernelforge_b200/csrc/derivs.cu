// Jacobian and Hessian FCHL19 local kernels (FP64 / FP32 arithmetic, with the
// contractions on tcgen05 tensor cores or through cuBLAS).
//
// Jacobian (+dK/dR of the "inner" set, src/local_kernels.cpp:791-974):
//   K[o, off_m + c] = sum_{j in m} v_{o,j} . J_j[:, c],
//   v_{o,j} = sum_{i in o, q_i = q_j} (e_ij / sigma^2) (x_i - x_j)
// The v rows are formed first (label-major register tiles on the CUDA cores,
// the squared distances from one dot-product GEMM per label), then contracted
// with the Jacobians, one GEMM problem per inner molecule m.  This costs
// 2 rep 3 n_m per (o, j) instead of per atom pair.  The transposed Jacobian
// (src/local_kernels.cpp:991-1166) is the same contraction with the roles of
// the sets swapped, negated and written transposed.
//
// Hessian (src/local_kernels.cpp:1171-1419):
//   H_ab = sum_{i in a} J_i^T Y_i,
//   Y_i  = sum_{j in b, q_j = q_i} (w_ij J_j - w'_ij d_ij (J_j^T d_ij)^T),
//   d_ij = x_i - x_j, w = e/sigma^2, w' = e/sigma^4
// t'_ij = w'_ij J_j^T d_ij is formed once per same-label atom pair (kernel 1,
// block per molecule pair; with tensor cores and FP32 inputs J_j^T d_ij is a
// difference of two projections of centred descriptors onto the Jacobian
// rows, one of them a tcgen05 GEMM per batch), Y_i per (pair, 8-row slice of
// rep) with the atoms of a label group in registers (kernel 2), and
// H_ab = J_a^T Y by one GEMM problem per pair, or per run of pairs
// (a, b), (a, b + 1), ... (tcgen05 split-fp16, or cuBLAS).  On that GEMM-form
// path (FP32, at most 64 atoms per molecule) Y_i keeps only sum_j w_ij J_j;
// the rank part -sum_ij (J_i^T d_ij) t'_ij^T is added to H_ab after the
// contraction by hess_rank_kernel, J_i^T d_ij coming from a third projection.
#include <cublas_v2.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <numeric>
#include <string>
#include <tuple>
#include <type_traits>

#include "derivs.h"
#include "kernels_common.cuh"
#include "tc_gemm.h"

namespace kfb {

kfb_status blas_for_stream(cudaStream_t s, cublasHandle_t *out);

namespace {

// --------------------------------------------------------- Jacobian: v rows
//   V[(o - o0) * NU + u, :] = sum_{i in o, q_i = q_u} w_iu (x_i - x_u)
//                           = sum_i w_iu x_i - (sum_i w_iu) x_u,
//   w_iu = exp(-|x_i - x_u|^2 / (2 sigma^2)) / sigma^2,
//   |x_i - x_u|^2 = |x_i|^2 + |x_u|^2 - 2 x_i . x_u (the dot products come
//   from one GEMM per label; the clamp at 0 absorbs rounding).
// Both atom sets are gathered label-major: inner atoms in sorted order su
// (runs [lab_start[l], lab_start[l+1])), outer atoms by (label, molecule),
// orng[o * nlab + l] = (first sorted row, count) of molecule o's label-l atoms.

// dst[r] = src[idx[r]] (rows of rep), norm[r] = |dst[r]|^2, *amax = max |dst|.
template <class T>
__global__ void gather_rows_norm_kernel(const T *__restrict__ src, const int *__restrict__ idx,
                                        int n, int rep, T *__restrict__ dst, T *__restrict__ norm,
                                        float *amax) {
    const int r = blockIdx.x;
    if (r >= n) return;
    const T *s = src + (size_t)idx[r] * rep;
    T *d = dst + (size_t)r * rep;
    T acc = T(0);
    float m = 0.f;
    for (int k = threadIdx.x; k < rep; k += blockDim.x) {
        const T v = s[k];
        d[k] = v;
        acc = fma(v, v, acc);
        m = fmaxf(m, fabsf((float)v));
    }
    __shared__ T red[8];
    __shared__ float redm[8];
    for (int o = 16; o; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[w] = acc;
        redm[w] = m;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        T t = T(0);
        float mm = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
            t += red[i];
            mm = fmaxf(mm, redm[i]);
        }
        norm[r] = t;
        // non-negative floats order like their bit patterns
        atomicMax(reinterpret_cast<int *>(amax), __float_as_int(mm));
    }
}

// hi/lo[r][k] = fp16 pair of src[r][k] * scale for k < rep, zero for
// rep <= k < kpad (K-major operands of the tensor-core dot products).
template <class T>
__global__ void split_pad_rows_kernel(const T *__restrict__ src, int rep, int kpad, float scale,
                                      __half *__restrict__ hi, __half *__restrict__ lo) {
    const size_t r = blockIdx.x;
    for (int k = threadIdx.x; k < kpad; k += blockDim.x) {
        const float v = k < rep ? (float)src[r * rep + k] * scale : 0.f;
        const __half h = __float2half_rn(v);
        hi[r * kpad + k] = h;
        lo[r * kpad + k] = __float2half_rn(v - __half2float(h));
    }
}

// Block per (outer molecule o = blockIdx.x, tile of up to JV_U sorted inner
// atoms of one label = blockIdx.y; consecutive blocks share the tile, whose
// rows then come from L2): 256 threads, each a 4 (atoms u) x 4 (consecutive
// k) register tile of a 64-wide pass over rep.  The block's weights
// (ns x JV_U, pre-multiplied by the output scale) and a slice of ks columns
// of o's label-l rows (ns x ks, ks a multiple of 64) sit in shared memory.
// Tiles of a label that o lacks write zero rows.  SPLIT writes the rows as
// the scaled fp16 pair (hi, lo) of the tensor-core contraction instead of T.
constexpr int JV_U = 64, JV_K = 64, JV_THREADS = 256;

template <class T>
__device__ __forceinline__ void ld4(const T *p, T (&v)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = *reinterpret_cast<const float4 *>(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    } else {
        const double2 a = *reinterpret_cast<const double2 *>(p);
        const double2 b = *reinterpret_cast<const double2 *>(p + 2);
        v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
    }
}

template <class T>
__device__ __forceinline__ void st4(T *p, const T (&v)[4]) {
    if constexpr (sizeof(T) == 4) {
        *reinterpret_cast<float4 *>(p) = make_float4(v[0], v[1], v[2], v[3]);
    } else {
        reinterpret_cast<double2 *>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2 *>(p)[1] = make_double2(v[2], v[3]);
    }
}

// (hi, lo) fp16 pairs of two values, hi = fp16(a), lo = fp16(a - hi)
__device__ __forceinline__ void split2(float a, float b, __half2 &hi, __half2 &lo) {
    hi = __floats2half2_rn(a, b);
    const float2 back = __half22float2(hi);
    lo = __floats2half2_rn(a - back.x, b - back.y);
}

template <class T, bool SPLIT>
__global__ void __launch_bounds__(JV_THREADS, sizeof(T) == 4 ? 3 : 2) jac_v_kernel(
    const int4 *__restrict__ tiles, const int2 *__restrict__ orng, int nlab, int o0,
    const long long *__restrict__ cinfo,
    const T *__restrict__ xo_s, const T *__restrict__ no_s, const T *__restrict__ xi_s,
    const T *__restrict__ ni_s, const T *__restrict__ D, const int *__restrict__ u_sorted,
    int NU, int rep, int lg_ks, T c2, T is2, T *__restrict__ V, __half *__restrict__ vh,
    __half *__restrict__ vl) {
    extern __shared__ __align__(16) unsigned char jv_raw[];
    const int4 tl = tiles[blockIdx.y];
    const int l = tl.x, u0 = tl.y, nu = tl.z - tl.y;
    const int ol = blockIdx.x;
    const int2 rg = orng[(size_t)(o0 + ol) * nlab + l];
    const int ns = rg.y;
    const int t = threadIdx.x;
    const bool vec = (rep & 3) == 0;
    if (ns == 0) {
        // o has no atom of this label: zero rows
        for (int uu = t >> 4; uu < nu; uu += JV_THREADS / 16) {
            const size_t row = ((size_t)ol * NU + u_sorted[u0 + uu]) * rep;
            for (int k = 4 * (t & 15); k < rep; k += 64) {
                if (vec) {
                    if constexpr (SPLIT) {
                        *reinterpret_cast<uint2 *>(vh + row + k) = make_uint2(0u, 0u);
                        *reinterpret_cast<uint2 *>(vl + row + k) = make_uint2(0u, 0u);
                    } else {
                        const T z[4] = {T(0), T(0), T(0), T(0)};
                        st4(V + row + k, z);
                    }
                } else {
                    for (int b = 0; b < 4 && k + b < rep; ++b) {
                        if constexpr (SPLIT) {
                            vh[row + k + b] = __float2half_rn(0.f);
                            vl[row + k + b] = __float2half_rn(0.f);
                        } else {
                            V[row + k + b] = T(0);
                        }
                    }
                }
            }
        }
        return;
    }
    const int ks = 1 << lg_ks;
    T *ws = reinterpret_cast<T *>(jv_raw);   // [ns][JV_U] weights
    T *xs = ws + (size_t)ns * JV_U;          // [ns][ks] slice of o's label-l rows
    T *wsum = xs + (size_t)ns * ks;          // [JV_U]
    {
        // dot products x_out . x_in: row (label block cinfo[l] + outer row offset),
        // column su, row stride NU
        const T *Dl = D + cinfo[l] + (long long)(rg.x - cinfo[nlab + l]) * NU + u0;
        for (int e = t; e < ns * JV_U; e += JV_THREADS) {
            const int r = e / JV_U, uu = e - r * JV_U;
            T w = T(0);
            if (uu < nu) {
                const T d2 = no_s[rg.x + r] + ni_s[u0 + uu] - T(2) * Dl[(size_t)r * NU + uu];
                w = kexp<T>(c2 * (d2 > T(0) ? d2 : T(0))) * is2;
            }
            ws[e] = w;
        }
        __syncthreads();
        if (t < JV_U) {
            T sum = T(0);
            for (int r = 0; r < ns; ++r) sum += ws[r * JV_U + t];
            wsum[t] = sum;
        }
        __syncthreads();
    }
    const int ug = t >> 4, kl = t & 15;   // atoms 4 ug .. 4 ug + 3, k = k0 + 4 kl ..
    // this thread's output rows, x_u rows and weight sums
    size_t orow[4];
    T sws[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const int uu = 4 * ug + a;
        orow[a] = ((size_t)ol * NU + (uu < nu ? u_sorted[u0 + uu] : 0)) * rep;
        sws[a] = wsum[uu];
    }
    const T *xu0 = xi_s + (size_t)(u0 + 4 * ug) * rep;
    const int nu_t = min(max(nu - 4 * ug, 0), 4);   // rows of this thread in the tile
    for (int s0 = 0; s0 < rep; s0 += ks) {
        if (s0 > 0) __syncthreads();   // previous slice consumed
        for (int e = t; e < (ns << lg_ks); e += JV_THREADS) {
            const int r = e >> lg_ks, kk = e & (ks - 1);
            xs[e] = (s0 + kk < rep) ? xo_s[(size_t)(rg.x + r) * rep + s0 + kk] : T(0);
        }
        __syncthreads();
        for (int kp = 0; kp < ks && s0 + kp < rep; kp += JV_K) {
            const int k = s0 + kp + 4 * kl;
            const bool full = vec && k + 3 < rep;
            // x_u of the epilogue, loaded ahead of the accumulation
            T xuv[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                const T *xu = xu0 + (size_t)a * rep + k;
                if (a < nu_t && full) {
                    ld4(xu, xuv[a]);
                } else {
#pragma unroll
                    for (int b = 0; b < 4; ++b) xuv[a][b] = (a < nu_t && k + b < rep) ? xu[b] : T(0);
                }
            }
            T acc[4][4];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
            const T *xr = xs + kp + 4 * kl;
            const T *wr = ws + 4 * ug;
#pragma unroll 2
            for (int r = 0; r < ns; ++r, xr += ks, wr += JV_U) {
                T xv[4], wv[4];
                ld4(xr, xv);
                ld4(wr, wv);
#pragma unroll
                for (int a = 0; a < 4; ++a)
#pragma unroll
                    for (int b = 0; b < 4; ++b) acc[a][b] = fma(wv[a], xv[b], acc[a][b]);
            }
            if (k >= rep) continue;
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                if (a >= nu_t) continue;
                const size_t row = orow[a] + k;
                T v[4];
#pragma unroll
                for (int b = 0; b < 4; ++b) v[b] = fma(-sws[a], xuv[a][b], acc[a][b]);
                if constexpr (SPLIT) {
                    __half2 h01, l01, h23, l23;
                    split2((float)v[0], (float)v[1], h01, l01);
                    split2((float)v[2], (float)v[3], h23, l23);
                    if (full) {
                        uint2 hv, lv;
                        hv.x = *reinterpret_cast<const unsigned *>(&h01);
                        hv.y = *reinterpret_cast<const unsigned *>(&h23);
                        lv.x = *reinterpret_cast<const unsigned *>(&l01);
                        lv.y = *reinterpret_cast<const unsigned *>(&l23);
                        *reinterpret_cast<uint2 *>(vh + row) = hv;
                        *reinterpret_cast<uint2 *>(vl + row) = lv;
                    } else {
                        const __half hh[4] = {__low2half(h01), __high2half(h01), __low2half(h23),
                                              __high2half(h23)};
                        const __half ll[4] = {__low2half(l01), __high2half(l01), __low2half(l23),
                                              __high2half(l23)};
                        for (int b = 0; b < 4 && k + b < rep; ++b) {
                            vh[row + b] = hh[b];
                            vl[row + b] = ll[b];
                        }
                    }
                } else {
                    if (full) {
                        st4(V + row, v);
                    } else {
                        for (int b = 0; b < 4 && k + b < rep; ++b) V[row + b] = v[b];
                    }
                }
            }
        }
    }
}

template <class T> struct BlasGemm;
template <> struct BlasGemm<float> {
    static cublasStatus_t run(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m,
                              int n, int k, const float *A, int lda, const float *B, int ldb,
                              float *C, int ldc) {
        const float one = 1.f, zero = 0.f;
        return cublasSgemm(h, ta, tb, m, n, k, &one, A, lda, B, ldb, &zero, C, ldc);
    }
};
template <> struct BlasGemm<double> {
    static cublasStatus_t run(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m,
                              int n, int k, const double *A, int lda, const double *B, int ldb,
                              double *C, int ldc) {
        const double one = 1.0, zero = 0.0;
        return cublasDgemm(h, ta, tb, m, n, k, &one, A, lda, B, ldb, &zero, C, ldc);
    }
};

// Label groups of a molecule pair: for each run [x, y) of equal labels in a's
// label order, the run [z, w) of the same label in b's (empty when b lacks
// it).  Returns the number of groups (<= na).
__device__ __forceinline__ int pair_label_groups(const int *la, const int *lb, int na, int nb,
                                                 int4 *groups) {
    int g = 0, t = 0;
    for (int s0 = 0; s0 < na;) {
        const int L = la[s0];
        int s1 = s0 + 1;
        while (s1 < na && la[s1] == L) ++s1;
        while (t < nb && lb[t] < L) ++t;
        int t1 = t;
        while (t1 < nb && lb[t1] == L) ++t1;
        groups[g++] = make_int4(s0, s1, t, t1);
        s0 = s1;
    }
    return g;
}

// N consecutive values from p, which is aligned to min(16, N sizeof(T)) bytes.
template <class T, int N>
__device__ __forceinline__ void load_vec(const T *p, T (&v)[N]) {
    if constexpr (sizeof(T) * N >= 16) {
        constexpr int per = 16 / sizeof(T);
#pragma unroll
        for (int q = 0; q < N / per; ++q) {
            const float4 f = reinterpret_cast<const float4 *>(p)[q];
            const T *e = reinterpret_cast<const T *>(&f);
#pragma unroll
            for (int r = 0; r < per; ++r) v[q * per + r] = e[r];
        }
    } else if constexpr (sizeof(T) * N == 8) {
        const float2 f = *reinterpret_cast<const float2 *>(p);
        const T *e = reinterpret_cast<const T *>(&f);
#pragma unroll
        for (int r = 0; r < N; ++r) v[r] = e[r];
    } else {
#pragma unroll
        for (int r = 0; r < N; ++r) v[r] = p[r];
    }
}

// Asynchronous global -> shared copies of one element (cp.async, L1-cached):
// each lane fetches its own words ahead of use, so a warp can stream rows of
// a Jacobian through a small ring without registers held for the prefetch.
template <class T>
__device__ __forceinline__ void cp_async_elem(T *smem, const T *gmem) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem));
    if constexpr (sizeof(T) == 4)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gmem));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
constexpr int JRING = 3;  // stages of the per-warp Jacobian ring

// Size of the balanced chunks of a label group of n atoms (at most cap each).
__device__ __forceinline__ int chunk_size(int n, int cap) {
    const int nch = (n + cap - 1) / cap;
    return (n + nch - 1) / nch;
}

// Largest of 1, 2, 4, ... that is <= n (n >= 1).
__device__ __forceinline__ int pow2_at_most(int n) {
    int p = 1;
    while (2 * p <= n) p <<= 1;
    return p;
}

// Smallest of 1, 2, 4, ... that is >= n.
__device__ __forceinline__ int pow2_at_least(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

// ------------------------------------------------------- Hessian kernel 1
// Block per molecule pair p = (a, b).  For every same-label atom pair (i, j):
//   W[p, i, j] = e_ij / sigma^2,
//   Tt[p, i, j, c] = (e_ij / sigma^4) (J_j^T (x_i - x_j))[c],  c < 3 n_b.
// Other (i, j) entries are not written (never read).  The weights come first
// (a warp per atom pair); then, per label group and balanced chunk of at most
// HT_IG atoms i of a (descriptors staged in shared memory), a warp item is (32
// columns, one partner j) accumulating the chunk's dot products over rep, so
// each J_j load feeds one FMA per atom of the chunk.  With a non-null bound
// the block raises *bound to an upper bound of |Y| (kernel 2's output) over
// its pair:  max_i [max|J_b| sum_j w_ij + sum_j |x_i - x_j|_inf |t'_ij|_inf]
// (|t'|_inf taken per 32-column slice and summed over the slices).
template <class T> struct HtCfg { static constexpr int IG = 16; };
template <> struct HtCfg<double> { static constexpr int IG = 8; };

__host__ __device__ inline size_t hess_t_head(int ma1, int ma2) {
    return ((size_t)ma1 * sizeof(int4) + (size_t)(ma1 + ma2 + ma1 + 1) * sizeof(int) +
            (size_t)(2 * ma1 + ma1 * ma2) * sizeof(float) + 15) &
           ~(size_t)15;
}

template <class T>
size_t hess_t_smem(int ma1, int ma2, int rep) {
    return hess_t_head(ma1, ma2) +
           ((size_t)HtCfg<T>::IG * ((rep + 7) & ~7) + (size_t)ma1 * ma2) * sizeof(T);
}

template <class T, int IGC, bool VEC>
__device__ __forceinline__ void ht_chunk(const T *__restrict__ xs, int rep8, int rep,
                                         const T *__restrict__ Jb, const T *__restrict__ xb,
                                         const int *pa, const int *pb, int4 gr, int i0, int cnt,
                                         int ncol, int ld2, size_t wbase, int ma2, const T *w2s,
                                         const float *dinf, float *bterm, T *__restrict__ Tt,
                                         T &jmax) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int nchunk = (ncol + 31) / 32;
    const int items = nchunk * (gr.w - gr.z);
    for (int it = warp; it < items; it += nwarp) {
        const int cc = it % nchunk, j = pb[gr.z + it / nchunk];
        const int c = cc * 32 + lane;
        const int cs = c < ncol ? c : 0;
        const T *Jj = Jb + (size_t)j * rep * ld2 + cs;
        const T *xj = xb + (size_t)j * rep;
        T acc[IGC];
#pragma unroll
        for (int ii = 0; ii < IGC; ++ii) acc[ii] = T(0);
        int k = 0;
        if (VEC) {
            for (; k + 8 <= rep; k += 8) {
                T jv[8], xv[8];
#pragma unroll
                for (int r = 0; r < 8; ++r) jv[r] = Jj[(size_t)(k + r) * ld2];
                load_vec<T, 8>(xj + k, xv);
#pragma unroll
                for (int r = 0; r < 8; ++r) jmax = fmax(jmax, fabs(jv[r]));
#pragma unroll
                for (int ii = 0; ii < IGC; ++ii) {
                    T xi[8];
                    load_vec<T, 8>(xs + ii * rep8 + k, xi);
#pragma unroll
                    for (int r = 0; r < 8; ++r) acc[ii] = fma(jv[r], xi[r] - xv[r], acc[ii]);
                }
            }
        }
        for (; k < rep; ++k) {
            const T jv = Jj[(size_t)k * ld2], xv = xj[k];
            jmax = fmax(jmax, fabs(jv));
#pragma unroll
            for (int ii = 0; ii < IGC; ++ii) acc[ii] = fma(jv, xs[ii * rep8 + k] - xv, acc[ii]);
        }
#pragma unroll
        for (int ii = 0; ii < IGC; ++ii) {
            if (ii < cnt) {
                const int i = pa[i0 + ii];
                const T t = w2s[i * ma2 + j] * acc[ii];
                if (c < ncol) Tt[(wbase + (size_t)i * ma2 + j) * ld2 + c] = t;
                if (bterm) {
                    float m = (c < ncol) ? fabsf((float)t) : 0.f;
                    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
                    if (lane == 0) atomicAdd(&bterm[i], dinf[i * ma2 + j] * m);
                }
            }
        }
    }
}

template <class T, bool VEC>
__global__ void __launch_bounds__(256) hess_t_kernel(
    const HessPair *__restrict__ pairs, const T *__restrict__ x1, const T *__restrict__ x2,
    const T *__restrict__ dx2, const int *__restrict__ perm1, const int *__restrict__ lab1,
    const int *__restrict__ perm2, const int *__restrict__ lab2, int ma1, int ma2, int rep,
    T c2, T is2, T is4, T *__restrict__ W, T *__restrict__ Tt, float *__restrict__ bound) {
    constexpr int IG = HtCfg<T>::IG;
    extern __shared__ __align__(16) unsigned char ht_raw[];
    int4 *groups = reinterpret_cast<int4 *>(ht_raw);  // ma1
    int *pa = reinterpret_cast<int *>(groups + ma1);   // ma1
    int *pb = pa + ma1;                                // ma2
    int *gstart = pb + ma2;                            // ma1 + 1: prefix of pair counts
    float *wsum = reinterpret_cast<float *>(gstart + ma1 + 1);  // ma1: sum_j w_ij
    float *bterm = wsum + ma1;                                   // ma1
    float *dinf = bterm + ma1;                                   // ma1 x ma2: |x_i - x_j|_inf
    const int rep8 = (rep + 7) & ~7;
    // xs first after the head: rows start on 16-byte boundaries (vector loads)
    T *xs = reinterpret_cast<T *>(ht_raw + hess_t_head(ma1, ma2));  // [IG][rep8]
    T *w2s = xs + (size_t)IG * rep8;                                  // [i][j] e / sigma^4
    __shared__ float red[8];
    __shared__ int ngroups;
    const int p = blockIdx.x;
    const HessPair pr = pairs[p];
    const int ld2 = 3 * ma2, ncol = 3 * pr.nb;
    const size_t wbase = (size_t)p * ma1 * ma2;
    for (int e = threadIdx.x; e < pr.na; e += blockDim.x) {
        pa[e] = perm1[(size_t)pr.a * ma1 + e];
        wsum[e] = 0.f;
        bterm[e] = 0.f;
    }
    for (int e = threadIdx.x; e < pr.nb; e += blockDim.x) pb[e] = perm2[(size_t)pr.b * ma2 + e];
    if (threadIdx.x == 0) {
        const int g = pair_label_groups(lab1 + (size_t)pr.a * ma1, lab2 + (size_t)pr.b * ma2,
                                        pr.na, pr.nb, groups);
        ngroups = g;
        gstart[0] = 0;
        for (int q = 0; q < g; ++q)
            gstart[q + 1] = gstart[q] + (groups[q].y - groups[q].x) * (groups[q].w - groups[q].z);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const T *xa = x1 + (size_t)pr.a * ma1 * rep, *xb = x2 + (size_t)pr.b * ma2 * rep;
    // weights of all same-label pairs
    for (int q = warp; q < gstart[ngroups]; q += nwarp) {
        int g = 0;
        while (gstart[g + 1] <= q) ++g;
        const int4 gr = groups[g];
        const int off = q - gstart[g], nbg = gr.w - gr.z;
        const int i = pa[gr.x + off / nbg], j = pb[gr.z + off % nbg];
        const T *xi = xa + (size_t)i * rep, *xj = xb + (size_t)j * rep;
        T dd = T(0), dm = T(0);
        for (int k = lane; k < rep; k += 32) {
            const T d = xi[k] - xj[k];
            dd = fma(d, d, dd);
            dm = fmax(dm, fabs(d));
        }
        for (int o = 16; o; o >>= 1) {
            dd += __shfl_xor_sync(0xffffffffu, dd, o);
            dm = fmax(dm, __shfl_xor_sync(0xffffffffu, dm, o));
        }
        if (lane == 0) {
            const T e = kexp<T>(c2 * dd);
            W[wbase + (size_t)i * ma2 + j] = e * is2;
            w2s[i * ma2 + j] = e * is4;
            dinf[i * ma2 + j] = (float)dm;
            if (bound) atomicAdd(&wsum[i], (float)(e * is2));
        }
    }
    const T *Jb = dx2 + (size_t)pr.b * ma2 * rep * ld2;
    T jmax = T(0);
    float *bt = bound ? bterm : nullptr;
    for (int g = 0; g < ngroups; ++g) {
        const int4 gr = groups[g];
        const int csz = chunk_size(gr.y - gr.x, IG);
        for (int i0 = gr.x; i0 < gr.y; i0 += csz) {
            const int cnt = min(csz, gr.y - i0);
            const int igc = pow2_at_least(cnt);
            __syncthreads();  // weights written / previous chunk's xs read
            for (int row = warp; row < igc; row += nwarp)
                for (int k = lane; k < rep8; k += 32)
                    xs[row * rep8 + k] =
                        (row < cnt && k < rep) ? xa[(size_t)pa[i0 + row] * rep + k] : T(0);
            __syncthreads();
            if (IG >= 16 && igc == 16)
                ht_chunk<T, (IG >= 16 ? 16 : 8), VEC>(xs, rep8, rep, Jb, xb, pa, pb, gr, i0, cnt,
                                                      ncol, ld2, wbase, ma2, w2s, dinf, bt, Tt,
                                                      jmax);
            else if (igc == 8)
                ht_chunk<T, 8, VEC>(xs, rep8, rep, Jb, xb, pa, pb, gr, i0, cnt, ncol, ld2, wbase,
                                    ma2, w2s, dinf, bt, Tt, jmax);
            else if (igc == 4)
                ht_chunk<T, 4, VEC>(xs, rep8, rep, Jb, xb, pa, pb, gr, i0, cnt, ncol, ld2, wbase,
                                    ma2, w2s, dinf, bt, Tt, jmax);
            else if (igc == 2)
                ht_chunk<T, 2, VEC>(xs, rep8, rep, Jb, xb, pa, pb, gr, i0, cnt, ncol, ld2, wbase,
                                    ma2, w2s, dinf, bt, Tt, jmax);
            else
                ht_chunk<T, 1, VEC>(xs, rep8, rep, Jb, xb, pa, pb, gr, i0, cnt, ncol, ld2, wbase,
                                    ma2, w2s, dinf, bt, Tt, jmax);
        }
    }
    if (!bound) return;
    // block max of |J_b| over the loaded rows, then max_i of the bound
    float jm = (float)jmax;
    for (int o = 16; o; o >>= 1) jm = fmaxf(jm, __shfl_xor_sync(0xffffffffu, jm, o));
    if (lane == 0) red[warp] = jm;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = lane < nwarp ? red[lane] : 0.f;
        for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        jm = v;
        float bmax = 0.f;
        for (int i = lane; i < pr.na; i += 32) bmax = fmaxf(bmax, jm * wsum[i] + bterm[i]);
        for (int o = 16; o; o >>= 1) bmax = fmaxf(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
        if (lane == 0) atomicMax(reinterpret_cast<int *>(bound), __float_as_int(bmax * 1.001f));
    }
}

template <class T>
kfb_status launch_hess_t(const HessPair *pairs, int np, const T *x1, const T *x2, const T *dx2,
                         const int *perm1, const int *lab1, const int *perm2, const int *lab2,
                         int ma1, int ma2, int rep, T c2, T is2, T is4, T *W, T *Tt,
                         float *bound, cudaStream_t s) {
    const size_t smem = hess_t_smem<T>(ma1, ma2, rep);
    if (smem > 200 * 1024)
        return set_error(KFB_ERR_INVALID_ARG, "max_atoms %d / %d, rep %d too large for the "
                         "Hessian kernel", ma1, ma2, rep);
    const bool vec = (rep % 8) == 0 && (reinterpret_cast<size_t>(x2) % 16) == 0;
    auto kern = vec ? hess_t_kernel<T, true> : hess_t_kernel<T, false>;
    if (smem > 48 * 1024)
        KFB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
    kern<<<np, 256, smem, s>>>(pairs, x1, x2, dx2, perm1, lab1, perm2, lab2, ma1, ma2, rep, c2,
                               is2, is4, W, Tt, bound);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

// ------------------------------------------ Hessian kernel 1, GEMM form (FP32)
// With tensor cores, J_j^T (x_i - x_j) comes from one product per batch of
// molecules b:  P[(a, i)][(b, j, c)] = (x_i - mu_l) . J_j[:, c]  (split fp16,
// tcgen05), and PB[(b, j, c)] = (x_j - mu_l) . J_j[:, c]  (FP64 sums), where
// mu_l is the set-1 mean of the label l both atoms share:
//   t_ij[c] = P[(a, i)][(b, j, c)] - PB[(b, j, c)].
// The centring keeps the two terms close to |J| |x - x_j| so that their
// difference loses little to cancellation.

// sums[l][k] += x[atom][k] over atoms of label index l (lidx < 0: skipped).
// Block (32 k, 8 atom groups); per-label partial sums in shared memory.
template <class T>
__global__ void __launch_bounds__(256) label_sums_kernel(const T *__restrict__ x,
                                                         const int *__restrict__ lidx, int natoms,
                                                         int rep, int L, double *__restrict__ sums) {
    extern __shared__ double ls[];   // [L][8][32]
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int k = blockIdx.x * 32 + tx;
    for (int e = threadIdx.x; e < L * 256; e += 256) ls[e] = 0.0;
    __syncthreads();
    for (int a = blockIdx.y * 8 + ty; a < natoms; a += gridDim.y * 8) {
        const int l = lidx[a];
        if (l >= 0 && k < rep) ls[(l * 8 + ty) * 32 + tx] += (double)x[(size_t)a * rep + k];
    }
    __syncthreads();
    if (ty == 0 && k < rep)
        for (int l = 0; l < L; ++l) {
            double sum = 0.0;
            for (int r = 0; r < 8; ++r) sum += ls[(l * 8 + r) * 32 + tx];
            atomicAdd(&sums[(size_t)l * rep + k], sum);
        }
}

// max |x - mu_l| over labelled atoms (FP32 bits, atomically)
template <class T>
__global__ void centred_absmax_kernel(const T *__restrict__ x, const int *__restrict__ lidx,
                                      int natoms, int rep, const double *__restrict__ sums,
                                      const double *__restrict__ inv_count, float *amax) {
    float m = 0.f;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
         e < (long long)natoms * rep; e += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(e / rep), k = (int)(e - (long long)a * rep);
        const int l = lidx[a];
        if (l < 0) continue;
        const double v = (double)x[e] - sums[(size_t)l * rep + k] * inv_count[l];
        m = fmaxf(m, fabsf((float)v));
    }
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(amax), __float_as_int(m));
}

// hi/lo[a][k] = fp16 pair of (x[a][k] - mu_l[k]) * scale; unlabelled rows zero;
// norm[a] = |x[a] - mu_l|^2 (FP64 sum).  Block (256) per row.
template <class T>
__global__ void __launch_bounds__(256) centred_split_kernel(
    const T *__restrict__ x, const int *__restrict__ lidx, int rep,
    const double *__restrict__ sums, const double *__restrict__ inv_count, float scale,
    __half *__restrict__ hi, __half *__restrict__ lo, float *__restrict__ norm) {
    const size_t a = blockIdx.x;
    const int l = lidx[a];
    double acc = 0.0;
    for (int k = threadIdx.x; k < rep; k += blockDim.x) {
        const double d = l < 0 ? 0.0 : (double)x[a * rep + k] - sums[(size_t)l * rep + k] *
                                                                    inv_count[l];
        acc = fma(d, d, acc);
        const float v = (float)(d * scale);
        const __half h = __float2half_rn(v);
        hi[a * rep + k] = h;
        lo[a * rep + k] = __float2half_rn(v - __half2float(h));
    }
    __shared__ double red[8];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += red[w];
        norm[a] = (float)t;
    }
}

// PB[(m, j)][c] = (x_j - mu_l) . J_j[:, c] (FP64 sums), block per atom (m, j)
template <class T>
__global__ void pb_kernel(const T *__restrict__ x2, const T *__restrict__ dx2,
                          const int *__restrict__ lidx2, int ma2, int rep,
                          const double *__restrict__ sums, const double *__restrict__ inv_count,
                          float *__restrict__ PB) {
    const size_t mj = blockIdx.x;
    const int ld2 = 3 * ma2;
    const int l = lidx2[mj];
    const T *xj = x2 + mj * rep;
    const T *J = dx2 + mj * rep * ld2;
    for (int c = threadIdx.x; c < ld2; c += blockDim.x) {
        double acc = 0.0;
        if (l >= 0)
            for (int k = 0; k < rep; ++k)
                acc = fma((double)xj[k] - sums[(size_t)l * rep + k] * inv_count[l],
                          (double)J[(size_t)k * ld2 + c], acc);
        PB[mj * ld2 + c] = (float)acc;
    }
}

// max |J_b| over the real atoms and columns of each molecule b (out zeroed
// first; blockIdx.y splits a molecule's rows, warps per row)
template <class T>
__global__ void jmax_per_mol_kernel(const T *__restrict__ dx, int ma, int rep,
                                    const int *__restrict__ nat, float *__restrict__ out) {
    const int m = blockIdx.x;
    const int na = min(max(nat[m], 0), ma), ld = 3 * ma, nc = 3 * na;
    const T *base = dx + (size_t)m * ma * rep * ld;
    float v = 0.f;
    const long long nrow = (long long)na * rep;
    const int nw = blockDim.x >> 5;
    for (long long row = (long long)blockIdx.y * nw + (threadIdx.x >> 5); row < nrow;
         row += (long long)gridDim.y * nw)
        for (int c = threadIdx.x & 31; c < nc; c += 32)
            v = fmaxf(v, fabsf((float)base[row * ld + c]));
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    // non-negative floats order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(out + m), __float_as_int(v));
}

// Kernel 1 with t from P: the same outputs as hess_t_kernel (W, Tt, bound;
// without the rank term in Y (rank_in_y = 0) the bound is max|J_b| sum_j w_ij);
// weights from the centred dot products G[(a, i)][(b - b0) * ma2 + j] (row
// length ldg) and the norms; t by a warp per (same-label pair, 32 columns).  P
// (row length ldp) holds the projections of same-label atoms only: atom (a, i)
// of molecules a0.. has row prow[(a - a0) ma1 + i], atom (b, j) of molecules
// b0.. the columns from pcol[(b - b0) ma2 + j] (its 3 ma2 coordinates).
__global__ void __launch_bounds__(256) hess_t_p_kernel(
    const HessPair *__restrict__ pairs, const float *__restrict__ G, long long ldg,
    const float *__restrict__ n1, const float *__restrict__ n2, const int *__restrict__ perm1,
    const int *__restrict__ lab1, const int *__restrict__ perm2, const int *__restrict__ lab2,
    int ma1, int ma2, float c2, float is2, float is4, const float *__restrict__ P,
    long long ldp, const int *__restrict__ prow, const int *__restrict__ pcol, int a0, int b0,
    const float *__restrict__ PB, const float *__restrict__ jbmax,
    int rank_in_y, float *__restrict__ W, float *__restrict__ Tt, float *__restrict__ bound) {
    extern __shared__ __align__(16) unsigned char ht_raw[];
    int4 *groups = reinterpret_cast<int4 *>(ht_raw);  // ma1
    int *pa = reinterpret_cast<int *>(groups + ma1);   // ma1
    int *pb = pa + ma1;                                // ma2
    int *gstart = pb + ma2;                            // ma1 + 1
    int *la = gstart + ma1 + 1;                        // ma1 (labels in sorted order)
    int *lb = la + ma1;                                // ma2
    float *wsum = reinterpret_cast<float *>(lb + ma2);  // ma1
    float *bterm = wsum + ma1;                          // ma1
    float *dinf = bterm + ma1;                          // ma1 x ma2
    float *w2s = dinf + (size_t)ma1 * ma2;              // ma1 x ma2
    __shared__ int ngroups;
    const int p = blockIdx.x;
    const HessPair pr = pairs[p];
    const int ld2 = 3 * ma2, ncol = 3 * pr.nb;
    const size_t wbase = (size_t)p * ma1 * ma2;
    for (int e = threadIdx.x; e < pr.na; e += blockDim.x) {
        pa[e] = perm1[(size_t)pr.a * ma1 + e];
        la[e] = lab1[(size_t)pr.a * ma1 + e];
        wsum[e] = 0.f;
        bterm[e] = 0.f;
    }
    for (int e = threadIdx.x; e < pr.nb; e += blockDim.x) {
        pb[e] = perm2[(size_t)pr.b * ma2 + e];
        lb[e] = lab2[(size_t)pr.b * ma2 + e];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int g = pair_label_groups(la, lb, pr.na, pr.nb, groups);
        ngroups = g;
        gstart[0] = 0;
        for (int q = 0; q < g; ++q)
            gstart[q + 1] = gstart[q] + (groups[q].y - groups[q].x) * (groups[q].w - groups[q].z);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int npairs = gstart[ngroups];
    auto pair_ij = [&](int q, int &i, int &j) {
        int g = 0;
        while (gstart[g + 1] <= q) ++g;
        const int4 gr = groups[g];
        const int off = q - gstart[g], nbg = gr.w - gr.z;
        i = pa[gr.x + off / nbg];
        j = pb[gr.z + off % nbg];
    };
    // weights of all same-label pairs (a thread per pair) from the centred dot
    // products g = (x_i - mu) . (x_j - mu) and norms:  |d|^2 = n_i + n_j - 2 g
    // (clamped at 0); |d|_2 bounds |d|_inf for the |Y| bound
    const float *Ga = G + (size_t)pr.a * ma1 * ldg + (size_t)(pr.b - b0) * ma2;
    for (int q = threadIdx.x; q < npairs; q += blockDim.x) {
        int i, j;
        pair_ij(q, i, j);
        const float dd = fmaxf(n1[(size_t)pr.a * ma1 + i] + n2[(size_t)pr.b * ma2 + j] -
                                   2.f * Ga[(size_t)i * ldg + j],
                               0.f);
        const float e = kexp<float>(c2 * dd);
        W[wbase + (size_t)i * ma2 + j] = e * is2;
        w2s[i * ma2 + j] = e * is4;
        dinf[i * ma2 + j] = sqrtf(dd);
        if (bound) atomicAdd(&wsum[i], e * is2);
    }
    __syncthreads();
    // t'_ij = w'_ij (P - PB), a warp per (pair, 32 columns)
    const int nchunk = (ncol + 31) / 32;
    const int *prow_a = prow + (size_t)(pr.a - a0) * ma1;
    const int *pcol_b = pcol + (size_t)(pr.b - b0) * ma2;
    const float *PBb = PB + (size_t)pr.b * ma2 * ld2;
    for (int it = warp; it < npairs * nchunk; it += nwarp) {
        const int q = it / nchunk, cc = it - q * nchunk;
        int i, j;
        pair_ij(q, i, j);
        const int c = cc * 32 + lane;
        float t = 0.f;
        if (c < ncol)
            t = w2s[i * ma2 + j] *
                (P[(size_t)prow_a[i] * ldp + pcol_b[j] + c] - PBb[(size_t)j * ld2 + c]);
        if (c < ncol) Tt[(wbase + (size_t)i * ma2 + j) * ld2 + c] = t;
        if (bound && rank_in_y) {
            float m = fabsf(t);
            for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
            if (lane == 0) atomicAdd(&bterm[i], dinf[i * ma2 + j] * m);
        }
    }
    if (!bound) return;
    __syncthreads();
    const float jm = jbmax[pr.b];
    if (warp == 0) {
        float bmax = 0.f;
        for (int i = lane; i < pr.na; i += 32) bmax = fmaxf(bmax, jm * wsum[i] + bterm[i]);
        for (int o = 16; o; o >>= 1) bmax = fmaxf(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
        if (lane == 0) atomicMax(reinterpret_cast<int *>(bound), __float_as_int(bmax * 1.001f));
    }
}

size_t hess_t_p_smem(int ma1, int ma2) {
    return (size_t)ma1 * sizeof(int4) + (size_t)(2 * ma1 + 2 * ma2 + ma1 + 1) * sizeof(int) +
           (size_t)(2 * ma1 + 2 * ma1 * ma2) * sizeof(float);
}

// ------------------------------------------------------- Hessian kernel 2
// Y_i = sum_j (w_ij J_j - w'_ij d_ij t_ij^T) for all atoms i of a, written as
//   Y_i[k, c] = sum_j (w_ij J_j[k, c] + x_j[k] t'_ij[c]) - x_i[k] r_i[c],
//   t'_ij = w'_ij t_ij (kernel 1 writes it scaled),  r_i = sum_j t'_ij
// over same-label atom pairs only.  Atoms of each molecule are visited in
// label order (perm: sorted position -> atom), so one label group of a meets
// one contiguous run of b.  Block per (pair, slice of kt rows of rep); each
// warp owns one (32 columns c, 8 rows k) tile and, for each label group and
// balanced chunk of at most HY_IG atoms i, keeps the chunk's 8 rows of Y in
// registers, so each J_j[k, c] load feeds two FMAs per atom of the chunk.
// Per partner j the warp streams J_j's tile, t'_ij[c] of the chunk and w_ij
// through a per-warp cp.async ring: no block-wide synchronisation after the
// descriptor rows of the slice are staged.
//   MODE 1: fp16 pair hi/lo of scale * Y, K-major rows (p, c) of (i, k)
//   MODE 2: Y[p, i, k, c] in T
//   MODE 3: as MODE 1 for Y_i = sum_j w_ij J_j alone (the rank term
//           -sum_j d_ij t'_ij^T is added to the Hessian block by
//           hess_rank_kernel after the contraction)
// FULL: rep % 8 == 0 (no row guards).
constexpr int HY_KR = 8;
template <class T> struct HyCfg { static constexpr int IG = 8, WARPS = 8; };
template <> struct HyCfg<double> { static constexpr int IG = 4, WARPS = 8; };
template <class T>
constexpr int hy_stage() {  // ring stage: J rows, t' of the chunk, w (one slot per lane)
    return (HY_KR + HyCfg<T>::IG + 1) * 32;
}

struct HyGeom {
    int kt;      // rows of rep per block (multiple of 8)
    int ldc;     // padded columns (multiple of 32)
    int warps;   // (ldc / 32) * (kt / 8)
    size_t smem;
};

template <class T>
HyGeom hess_y_geom(int ma1, int ma2) {
    HyGeom g;
    const int nchunk = (3 * ma2 + 31) / 32;
    const int kgroups = std::max(1, HyCfg<T>::WARPS / nchunk);
    g.kt = 8 * kgroups;
    g.ldc = 32 * nchunk;
    g.warps = nchunk * kgroups;
    const size_t head =
        ((size_t)ma1 * sizeof(int4) + (size_t)2 * (ma1 + ma2) * sizeof(int) + 15) & ~(size_t)15;
    g.smem = head + ((size_t)(ma1 + ma2) * g.kt + (size_t)g.warps * JRING * hy_stage<T>()) *
                        sizeof(T);
    return g;
}

// One chunk of exactly IGC atoms (i0 .. i0 + IGC - 1 in label order) of group gr.
template <class T, int IGC, int MODE, bool FULL>
__device__ __forceinline__ void hy_chunk(const HessPair &pr, int p, int4 gr, int i0,
                                         const int *pa, const int *pb, const T *xa_s,
                                         const T *xb_s, T *ring, int kt, int ma1, int ma2,
                                         int rep, int k0, int kk0, int c,
                                         const T *__restrict__ dx2, const T *__restrict__ W,
                                         const T *__restrict__ Tt, float scale,
                                         __half *__restrict__ yhi, __half *__restrict__ ylo,
                                         T *__restrict__ Y) {
    constexpr int IG = HyCfg<T>::IG, SS = hy_stage<T>();
    constexpr bool RANK = MODE != 3;
    const int lane = threadIdx.x & 31;
    const int ld2 = 3 * ma2, ncol = 3 * pr.nb;
    const int cs = c < ncol ? c : 0;
    const size_t wbase = (size_t)p * ma1 * ma2;
    T acc[IGC][HY_KR], rr[IGC];
#pragma unroll
    for (int ii = 0; ii < IGC; ++ii) {
        rr[ii] = T(0);
#pragma unroll
        for (int r = 0; r < HY_KR; ++r) acc[ii][r] = T(0);
    }
    const T *Jb = dx2 + ((size_t)pr.b * ma2 * rep + k0) * (size_t)ld2 + cs;
    const T *Tb = Tt + wbase * ld2 + cs;
    const T *Wb = W + wbase;
    const int nj = gr.w - gr.z;
    auto issue = [&](int jj, int stage) {
        if (jj < nj) {
            const int j = pb[gr.z + jj];
            T *dst = ring + stage * SS;
            const T *Jj = Jb + (size_t)j * rep * ld2;
#pragma unroll
            for (int r = 0; r < HY_KR; ++r) {
                if (FULL || k0 + r < rep)
                    cp_async_elem<T>(dst + r * 32 + lane, Jj + (size_t)r * ld2);
                else
                    dst[r * 32 + lane] = T(0);
            }
            if (RANK) {
#pragma unroll
                for (int ii = 0; ii < IGC; ++ii)
                    cp_async_elem<T>(dst + (HY_KR + ii) * 32 + lane,
                                     Tb + ((size_t)pa[i0 + ii] * ma2 + j) * ld2);
            }
            // lane l fetches w of atom l mod IGC (no divergent branch)
            cp_async_elem<T>(dst + (HY_KR + IG) * 32 + lane,
                             Wb + (size_t)pa[i0 + (lane & (IGC - 1))] * ma2 + j);
        }
        cp_async_commit();
    };
    issue(0, 0);
    issue(1, 1);
    int st = 0;
    for (int jj = 0; jj < nj; ++jj) {
        issue(jj + 2, st == 0 ? 2 : st - 1);
        cp_async_wait<JRING - 1>();
        // every lane reads only the ring slots it filled itself; w_ij of the
        // chunk (fetched by lanes 0..IGC-1) is broadcast by shuffles
        const T *src = ring + st * SS;
        T jv[HY_KR], xj[HY_KR], t[IGC], w[IGC];
#pragma unroll
        for (int r = 0; r < HY_KR; ++r) jv[r] = src[r * 32 + lane];
        const T wl = src[(HY_KR + IG) * 32 + lane];
#pragma unroll
        for (int ii = 0; ii < IGC; ++ii) {
            if (RANK) t[ii] = src[(HY_KR + ii) * 32 + lane];
            w[ii] = __shfl_sync(0xffffffffu, wl, ii);
        }
        if (RANK) load_vec<T, HY_KR>(xb_s + pb[gr.z + jj] * kt + kk0, xj);
        st = st == JRING - 1 ? 0 : st + 1;
#pragma unroll
        for (int ii = 0; ii < IGC; ++ii) {
            if (RANK) {
                rr[ii] += t[ii];
#pragma unroll
                for (int r = 0; r < HY_KR; ++r)
                    acc[ii][r] = fma(w[ii], jv[r], fma(xj[r], t[ii], acc[ii][r]));
            } else {
#pragma unroll
                for (int r = 0; r < HY_KR; ++r) acc[ii][r] = fma(w[ii], jv[r], acc[ii][r]);
            }
        }
    }
    if (c >= ncol) return;
#pragma unroll
    for (int ii = 0; ii < IGC; ++ii) {
        const int i = pa[i0 + ii];
        if (RANK) {
            T xi[HY_KR];
            load_vec<T, HY_KR>(xa_s + i * kt + kk0, xi);
#pragma unroll
            for (int r = 0; r < HY_KR; ++r) acc[ii][r] = fma(-xi[r], rr[ii], acc[ii][r]);
        }
        if (MODE != 2) {
            // rep % 16 == 0 on this path: 8 rows are 16 aligned bytes
            // packed conversions: two values per instruction
            unsigned hw[HY_KR / 2], lw[HY_KR / 2];
#pragma unroll
            for (int r = 0; r < HY_KR; r += 2) {
                const float2 v = make_float2((float)acc[ii][r] * scale,
                                             (float)acc[ii][r + 1] * scale);
                const __half2 h = __float22half2_rn(v);
                const float2 hf = __half22float2(h);
                const __half2 l = __float22half2_rn(make_float2(v.x - hf.x, v.y - hf.y));
                hw[r / 2] = *reinterpret_cast<const unsigned *>(&h);
                lw[r / 2] = *reinterpret_cast<const unsigned *>(&l);
            }
            const size_t o = (((size_t)p * ld2 + c) * ma1 + i) * (size_t)rep + k0;
            *reinterpret_cast<uint4 *>(yhi + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(ylo + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        } else {
            T *Yi = Y + ((size_t)p * ma1 + i) * rep * (size_t)ld2 + c;
#pragma unroll
            for (int r = 0; r < HY_KR; ++r)
                if (FULL || k0 + r < rep) Yi[(size_t)(k0 + r) * ld2] = acc[ii][r];
        }
    }
}

template <class T, int MODE, bool FULL>
__global__ void __launch_bounds__(256, 2) hess_y_kernel(
    const HessPair *__restrict__ pairs, const T *__restrict__ x1, const T *__restrict__ x2,
    const T *__restrict__ dx2, const int *__restrict__ perm1, const int *__restrict__ lab1,
    const int *__restrict__ perm2, const int *__restrict__ lab2, int ma1, int ma2, int rep,
    int kt, int ldc, const T *__restrict__ W, const T *__restrict__ Tt, float scale,
    __half *__restrict__ yhi, __half *__restrict__ ylo, T *__restrict__ Y) {
    constexpr int IG = HyCfg<T>::IG;
    extern __shared__ __align__(16) unsigned char hy_raw[];
    int4 *groups = reinterpret_cast<int4 *>(hy_raw);  // ma1
    int *pa = reinterpret_cast<int *>(groups + ma1);   // ma1
    int *pb = pa + ma1;                                // ma2
    int *la = pb + ma2;                                // ma1 (labels in sorted order)
    int *lb = la + ma1;                                // ma2
    T *xa_s = reinterpret_cast<T *>(
        hy_raw + (((size_t)ma1 * sizeof(int4) + (size_t)2 * (ma1 + ma2) * sizeof(int) + 15) &
                  ~(size_t)15));
    T *xb_s = xa_s + (size_t)ma1 * kt;      // [atom][row of the slice]
    T *jring = xb_s + (size_t)ma2 * kt;     // per warp [JRING][stage]
    __shared__ int ngroups;
    const int p = blockIdx.y;
    const HessPair pr = pairs[p];
    const int kbase = blockIdx.x * kt;
    for (int e = threadIdx.x; e < pr.na; e += blockDim.x) {
        pa[e] = perm1[(size_t)pr.a * ma1 + e];
        la[e] = lab1[(size_t)pr.a * ma1 + e];
    }
    for (int e = threadIdx.x; e < pr.nb; e += blockDim.x) {
        pb[e] = perm2[(size_t)pr.b * ma2 + e];
        lb[e] = lab2[(size_t)pr.b * ma2 + e];
    }
    if (MODE != 3) {  // descriptor rows of the slice (rank term)
        for (int e = threadIdx.x; e < pr.na * kt; e += blockDim.x) {
            const int i = e / kt, kk = e - i * kt;
            xa_s[e] = (kbase + kk < rep) ? x1[((size_t)pr.a * ma1 + i) * rep + kbase + kk] : T(0);
        }
        for (int e = threadIdx.x; e < pr.nb * kt; e += blockDim.x) {
            const int j = e / kt, kk = e - j * kt;
            xb_s[e] = (kbase + kk < rep) ? x2[((size_t)pr.b * ma2 + j) * rep + kbase + kk] : T(0);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0)  // atoms of a whose label b lacks get Y = 0 (written)
        ngroups = pair_label_groups(la, lb, pr.na, pr.nb, groups);
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nchunk = ldc / 32;
    const int kk0 = (warp / nchunk) * HY_KR, k0 = kbase + kk0;
    if (k0 >= rep) return;  // warp-uniform; no block-wide synchronisation follows
    const int c = (warp % nchunk) * 32 + lane;
    T *ring = jring + (size_t)warp * JRING * hy_stage<T>();
    for (int g = 0; g < ngroups; ++g) {
        const int4 gr = groups[g];
        // chunks of power-of-two sizes (largest first): no padded FMAs
        for (int i0 = gr.x, cnt; i0 < gr.y; i0 += cnt) {
            cnt = pow2_at_most(min(IG, gr.y - i0));
            const int igc = cnt;
#define KFB_HY_CHUNK(N)                                                                       \
    hy_chunk<T, N, MODE, FULL>(pr, p, gr, i0, pa, pb, xa_s, xb_s, ring, kt, ma1, ma2, rep, \
                               k0, kk0, c, dx2, W, Tt, scale, yhi, ylo, Y)
            if (IG >= 8 && igc == 8)
                KFB_HY_CHUNK((IG >= 8 ? 8 : 4));
            else if (igc == 4)
                KFB_HY_CHUNK(4);
            else if (igc == 2)
                KFB_HY_CHUNK(2);
            else
                KFB_HY_CHUNK(1);
#undef KFB_HY_CHUNK
        }
    }
}

// ------------------------------------------------------- Hessian rank term
// With Y_i = sum_j w_ij J_j (MODE 3) the contraction leaves out
//   -sum_i J_i^T sum_j d_ij t'_ij^T = -sum_{i, j same label} s_ij t'_ij^T,
//   s_ij[c'] = J_i[:, c'] . (x_i - x_j) = PB1[(a, i)][c'] - Q[qrow(b, j)][qcol(a, i) + c'],
// PB1 = (x_i - mu_l) . J_i[:, c'] and Q = (x_j - mu_l) . J_i[:, c'] (one
// projection GEMM problem per label and batch over the label's atoms of the
// batch's molecules b and the Jacobian rows of its atoms in the batch's
// molecules a; mu_l the label centre that also centres P).  qrow / qcol map
// atoms of molecules b0.. / a0.. to their row / first column of Q.  This kernel adds that term to the pair's Hessian block after
// the contraction wrote it: block per (pair, 64 x 64 tile of (c', c)),
// 256 threads of 4 x 4 register tiles, the same-label pairs in chunks of HR_Q
// with their s and t' rows staged in shared memory.  Every output element
// belongs to one thread of one block and the contraction ran before on the
// same stream, so the adds need no atomics.  ma1, ma2 <= HR_MAXA.
constexpr int HR_Q = 32, HR_T = 64, HR_MAXA = 64;
__global__ void __launch_bounds__(256) hess_rank_kernel(
    const HessPair *__restrict__ pairs, const int *__restrict__ perm1,
    const int *__restrict__ lab1, const int *__restrict__ perm2, const int *__restrict__ lab2,
    int ma1, int ma2, const float *__restrict__ Q, long long ldq, const int *__restrict__ qrow,
    const int *__restrict__ qcol, int a0, int b0, const float *__restrict__ PB1, const float *__restrict__ Tt, const int *__restrict__ off1,
    const int *__restrict__ off2, int symmetric, ElemSink sink) {
    __shared__ int4 groups[HR_MAXA];
    __shared__ int pa[HR_MAXA], pb[HR_MAXA], la[HR_MAXA], lb[HR_MAXA], gstart[HR_MAXA + 1];
    __shared__ int qi[HR_Q], qj[HR_Q];
    __shared__ int ngroups;
    __shared__ __align__(16) float Ss[HR_Q][HR_T];
    __shared__ __align__(16) float Ts[HR_Q][HR_T];
    const int p = blockIdx.y;
    const HessPair pr = pairs[p];
    const int ld1 = 3 * ma1, ld2 = 3 * ma2, m1 = 3 * pr.na, n2 = 3 * pr.nb;
    const int ntc = (ld2 + HR_T - 1) / HR_T;
    const int r0 = (blockIdx.x / ntc) * HR_T, c0 = (blockIdx.x % ntc) * HR_T;
    if (r0 >= m1 || c0 >= n2) return;  // block-uniform
    const int tid = threadIdx.x;
    for (int e = tid; e < pr.na; e += blockDim.x) {
        pa[e] = perm1[(size_t)pr.a * ma1 + e];
        la[e] = lab1[(size_t)pr.a * ma1 + e];
    }
    for (int e = tid; e < pr.nb; e += blockDim.x) {
        pb[e] = perm2[(size_t)pr.b * ma2 + e];
        lb[e] = lab2[(size_t)pr.b * ma2 + e];
    }
    __syncthreads();
    if (tid == 0) {
        const int g = pair_label_groups(la, lb, pr.na, pr.nb, groups);
        ngroups = g;
        gstart[0] = 0;
        for (int q = 0; q < g; ++q)
            gstart[q + 1] = gstart[q] + (groups[q].y - groups[q].x) * (groups[q].w - groups[q].z);
    }
    __syncthreads();
    const int npairs = gstart[ngroups];
    const int ty = tid >> 4, tx = tid & 15;
    const size_t arow = (size_t)pr.a * ma1;
    const int *qrow_b = qrow + (size_t)(pr.b - b0) * ma2;
    const int *qcol_a = qcol + (size_t)(pr.a - a0) * ma1;
    const float *Tp = Tt + (size_t)p * ma1 * ma2 * ld2;
    float acc[4][4] = {};
    for (int q0 = 0; q0 < npairs; q0 += HR_Q) {
        if (tid < HR_Q) {
            const int q = q0 + tid;
            int i = -1, j = -1;
            if (q < npairs) {
                int g = 0;
                while (gstart[g + 1] <= q) ++g;
                const int4 gr = groups[g];
                const int off = q - gstart[g], nbg = gr.w - gr.z;
                i = pa[gr.x + off / nbg];
                j = pb[gr.z + off % nbg];
            }
            qi[tid] = i;
            qj[tid] = j;
        }
        __syncthreads();
        for (int e = tid; e < HR_Q * HR_T; e += blockDim.x) {
            const int qq = e / HR_T, r = e - qq * HR_T;
            const int i = qi[qq], j = qj[qq];
            float sv = 0.f, tv = 0.f;
            if (i >= 0) {
                const size_t col = (arow + i) * ld1;
                if (r0 + r < m1)
                    sv = PB1[col + r0 + r] - Q[(size_t)qrow_b[j] * ldq + qcol_a[i] + r0 + r];
                if (c0 + r < n2) tv = Tp[((size_t)i * ma2 + j) * ld2 + c0 + r];
            }
            Ss[qq][r] = sv;
            Ts[qq][r] = tv;
        }
        __syncthreads();
#pragma unroll 8
        for (int qq = 0; qq < HR_Q; ++qq) {
            const float4 sv = *reinterpret_cast<const float4 *>(&Ss[qq][ty * 4]);
            const float4 tv = *reinterpret_cast<const float4 *>(&Ts[qq][tx * 4]);
            const float sa[4] = {sv.x, sv.y, sv.z, sv.w}, ta[4] = {tv.x, tv.y, tv.z, tv.w};
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(sa[u], ta[v], acc[u][v]);
        }
        __syncthreads();  // Ss, Ts, qi, qj reused
    }
    const int dg = (symmetric && pr.a == pr.b) ? 1 : 0;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int R = r0 + ty * 4 + u;
        if (R >= m1) continue;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int C = c0 + tx * 4 + v;
            if (C >= n2) continue;
            const double val = -(double)acc[u][v];
            sink_positions(sink, (long long)off1[pr.a] + R, (long long)off2[pr.b] + C, dg,
                           [&](long long idx) { sink_add(sink, idx, val); });
        }
    }
}

// ------------------------------------------------- Y on the tensor cores
// Without the rank term, Y_p[(c, k)][i] = sum_j W_p[i][j] J_b[j][k][c] is one
// GEMM per molecule b over the batch's pairs that share it: A = the Jacobian
// of b with rows (c, k) and the atoms j as K (jk_split_kernel, once per call),
// B = the pairs' weight rows (p, i) in b order (w_split_kernel, per batch),
// and the grouped GEMM's EPI_YSPLIT epilogue writes the fp16 pair of Y where
// the contraction reads it.  K = kj = ma2 rounded up to 16; entries of atoms
// j >= n_b are zero in A, entries of other-label pairs are zero in W.

// Jk[((b ld + c) rep + k) kj + j] = scale * dX[b][j][k][c] as an fp16 pair,
// rows c < 3 n_b; block per (k, b), eight atoms j per pass.
template <class T>
__global__ void __launch_bounds__(128) jk_split_kernel(const T *__restrict__ dx, int ma, int rep,
                                                       int kj, const int *__restrict__ nat,
                                                       float scale, __half *__restrict__ hi,
                                                       __half *__restrict__ lo) {
    extern __shared__ float jk_s[];  // [8][ld + 1]
    const int k = blockIdx.x, b = blockIdx.y;
    const int nb = min(max(nat[b], 0), ma), ld = 3 * ma, nc = 3 * nb;
    for (int j0 = 0; j0 < kj; j0 += 8) {
        __syncthreads();
        for (int e = threadIdx.x; e < 8 * nc; e += blockDim.x) {
            const int r = e / nc, c = e - r * nc, j = j0 + r;
            jk_s[r * (ld + 1) + c] =
                j < nb ? (float)dx[(((size_t)b * ma + j) * rep + k) * ld + c] * scale : 0.f;
        }
        __syncthreads();
        for (int c = threadIdx.x; c < nc; c += blockDim.x) {
            unsigned hw[4], lw[4];
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const float2 v = make_float2(jk_s[r * (ld + 1) + c], jk_s[(r + 1) * (ld + 1) + c]);
                const __half2 h = __float22half2_rn(v);
                const float2 hf = __half22float2(h);
                const __half2 l = __float22half2_rn(make_float2(v.x - hf.x, v.y - hf.y));
                hw[r / 2] = *reinterpret_cast<const unsigned *>(&h);
                lw[r / 2] = *reinterpret_cast<const unsigned *>(&l);
            }
            const size_t o = (((size_t)b * ld + c) * rep + k) * (size_t)kj + j0;
            *reinterpret_cast<uint4 *>(hi + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
            *reinterpret_cast<uint4 *>(lo + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        }
    }
}

// Ws[r kj + j] = scale * W[border[q]][i][j] (r = q ma1 + i) as an fp16 pair,
// zero for j >= ma2; a thread per (row, eight columns).
__global__ void w_split_kernel(const float *__restrict__ W, const int *__restrict__ border,
                               int nrows, int ma1, int ma2, int kj, float scale,
                               __half *__restrict__ hi, __half *__restrict__ lo) {
    const int ng = kj / 8;
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (long long)nrows * ng) return;
    const int r = (int)(e / ng), j0 = (int)(e - (long long)r * ng) * 8;
    const int q = r / ma1, i = r - q * ma1;
    const float *w = W + ((size_t)border[q] * ma1 + i) * ma2;
    unsigned hw[4], lw[4];
#pragma unroll
    for (int u = 0; u < 8; u += 2) {
        const float2 v = make_float2(j0 + u < ma2 ? w[j0 + u] * scale : 0.f,
                                     j0 + u + 1 < ma2 ? w[j0 + u + 1] * scale : 0.f);
        const __half2 h = __float22half2_rn(v);
        const float2 hf = __half22float2(h);
        const __half2 l = __float22half2_rn(make_float2(v.x - hf.x, v.y - hf.y));
        hw[u / 2] = *reinterpret_cast<const unsigned *>(&h);
        lw[u / 2] = *reinterpret_cast<const unsigned *>(&l);
    }
    const size_t o = (size_t)r * kj + j0;
    *reinterpret_cast<uint4 *>(hi + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
    *reinterpret_cast<uint4 *>(lo + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
}

template <class T, int MODE>
kfb_status launch_hess_y(const HessPair *pairs, int np, const T *x1, const T *x2, const T *dx2,
                         const int *perm1, const int *lab1, const int *perm2, const int *lab2,
                         int ma1, int ma2, int rep, const T *W, const T *Tt, float scale,
                         __half *yhi, __half *ylo, T *Y, cudaStream_t s) {
    const HyGeom g = hess_y_geom<T>(ma1, ma2);
    if (g.warps > 8 || g.smem > 100 * 1024)
        return set_error(KFB_ERR_INVALID_ARG, "max_atoms %d / %d too large for the Hessian kernel",
                         ma1, ma2);
    const bool full = rep % 8 == 0;
    auto kern = full ? hess_y_kernel<T, MODE, true> : hess_y_kernel<T, MODE, false>;
    if (g.smem > 48 * 1024)
        KFB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)g.smem));
    const dim3 grid((unsigned)((rep + g.kt - 1) / g.kt), (unsigned)np);
    kern<<<grid, 32 * g.warps, g.smem, s>>>(pairs, x1, x2, dx2, perm1, lab1, perm2, lab2, ma1,
                                            ma2, rep, g.kt, g.ldc, W, Tt, scale, yhi, ylo, Y);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

// Atoms of every molecule in label order: perm[m * ma + s] = atom at sorted
// position s, lab[m * ma + s] its label (stable within a label).
void label_order(const SetView &v, std::vector<int> &perm, std::vector<int> &lab) {
    perm.assign((size_t)v.nm * v.ma, 0);
    lab.assign((size_t)v.nm * v.ma, 0);
    std::vector<int> idx;
    for (int m = 0; m < v.nm; ++m) {
        const int n = v.natoms(m);
        const int32_t *q = v.q + (size_t)m * v.ma;
        idx.resize(n);
        for (int i = 0; i < n; ++i) idx[i] = i;
        std::stable_sort(idx.begin(), idx.end(), [&](int x, int y) { return q[x] < q[y]; });
        for (int s2 = 0; s2 < n; ++s2) {
            perm[(size_t)m * v.ma + s2] = idx[s2];
            lab[(size_t)m * v.ma + s2] = q[idx[s2]];
        }
    }
}

// Contractions on CUDA cores through cuBLAS: problems of equal shape run as
// one batched GEMM into a scratch array, then a scatter kernel writes each
// result through the sink (alpha applied there).  Row-major
// C (M x N) = A' (M x K) B (K x N) is the column-major C^T = B^T A'^T.
template <class T> struct BlasBatched;
template <> struct BlasBatched<float> {
    static cublasStatus_t run(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m,
                              int n, int k, const float *const A[], int lda,
                              const float *const B[], int ldb, float *const C[], int ldc,
                              int cnt) {
        const float one = 1.f, zero = 0.f;
        return cublasSgemmBatched(h, ta, tb, m, n, k, &one, A, lda, B, ldb, &zero, C, ldc, cnt);
    }
};
template <> struct BlasBatched<double> {
    static cublasStatus_t run(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, int m,
                              int n, int k, const double *const A[], int lda,
                              const double *const B[], int ldb, double *const C[], int ldc,
                              int cnt) {
        const double one = 1.0, zero = 0.0;
        return cublasDgemmBatched(h, ta, tb, m, n, k, &one, A, lda, B, ldb, &zero, C, ldc, cnt);
    }
};

struct ScatterProb {
    long long coff;
    int M, N, row_off, col_off, diag, pad;
    double alpha;
};

template <class T>
__global__ void scatter_sink_kernel(const ScatterProb *__restrict__ probs, const T *__restrict__ C,
                                    ElemSink sink) {
    const ScatterProb sp = probs[blockIdx.x];
    for (int e = threadIdx.x; e < sp.M * sp.N; e += blockDim.x) {
        const int m = e / sp.N, n = e - m * sp.N;
        sink_store(sink, sp.row_off + m, sp.col_off + n, (double)C[sp.coff + e] * sp.alpha,
                   sp.diag);
    }
}

template <class T>
kfb_status launch_gemm(const std::vector<GemmProb> &probs, const ElemSink &sink,
                       cudaStream_t s) {
    const int n = (int)probs.size();
    if (n == 0) return KFB_OK;
    cublasHandle_t h = nullptr;
    KFB_TRY(blas_for_stream(s, &h));
    auto key = [&](int q) {
        const GemmProb &g = probs[q];
        return std::make_tuple(g.transA, g.M, g.N, g.K, g.lda, g.ldb);
    };
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return key(x) < key(y); });
    std::vector<ScatterProb> sp(n);
    long long total = 0;
    for (int q = 0; q < n; ++q) {
        const GemmProb &g = probs[order[q]];
        sp[q] = ScatterProb{total, g.M, g.N, g.row_off, g.col_off, g.diag, 0, g.alpha};
        total += (long long)g.M * g.N;
    }
    DevBuf C, ptrs, dsp;
    KFB_TRY(C.alloc((size_t)std::max<long long>(total, 1) * sizeof(T), s));
    std::vector<const void *> pv(3 * (size_t)n);
    for (int q = 0; q < n; ++q) {
        const GemmProb &g = probs[order[q]];
        pv[q] = g.A;
        pv[n + q] = g.B;
        pv[2 * n + q] = C.as<T>() + sp[q].coff;
    }
    KFB_TRY(upload(ptrs, pv, s));
    KFB_TRY(upload(dsp, sp, s));
    void **base = static_cast<void **>(ptrs.ptr);
    const T *const *dA = reinterpret_cast<const T *const *>(base);
    const T *const *dB = dA + n;
    T *const *dC = reinterpret_cast<T *const *>(base + 2 * (size_t)n);
    for (int q0 = 0; q0 < n;) {
        int q1 = q0 + 1;
        while (q1 < n && key(order[q1]) == key(order[q0])) ++q1;
        const GemmProb &g = probs[order[q0]];
        if (g.M > 0 && g.N > 0 && g.K > 0) {
            const cublasStatus_t st = BlasBatched<T>::run(
                h, CUBLAS_OP_N, g.transA ? CUBLAS_OP_T : CUBLAS_OP_N, g.N, g.M, g.K, dB + q0,
                (int)g.ldb, dA + q0, (int)g.lda, dC + q0, g.N, q1 - q0);
            if (st != CUBLAS_STATUS_SUCCESS)
                return set_error(KFB_ERR_CUDA, "batched GEMM failed: cublas status %d", (int)st);
        } else {
            KFB_TRY(zero(C.as<T>() + sp[q0].coff,
                         (size_t)(sp[q1 - 1].coff + (long long)sp[q1 - 1].M * sp[q1 - 1].N -
                                  sp[q0].coff) * sizeof(T), s));
        }
        q0 = q1;
    }
    scatter_sink_kernel<T><<<n, 256, 0, s>>>(dsp.as<ScatterProb>(), C.as<T>(), sink);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

size_t budget_bytes() {
    const char *env = getenv("KFB_WORKSPACE_GB");
    double gb = env ? atof(env) : 4.0;
    if (!(gb > 0.0)) gb = 4.0;
    return (size_t)(gb * 1073741824.0);
}

}  // namespace

// ---------------------------------------------------------------------------
// Jacobian core: G[o, off_in[m] + c] (through `sink`, scaled by alpha) for all
// outer molecules o and inner molecules m.
// ---------------------------------------------------------------------------
template <class T>
kfb_status jacobian_core(const DerivSet &outer, const DerivSet &inner, int rep, double sigma,
                         double alpha, bool tc, ElemSink sink, cudaStream_t s) {
    std::vector<int> in_offs;
    deriv_offsets(inner.v, in_offs);
    // active inner atoms in molecule order
    std::vector<int> u_src, u_lab, u_first(inner.v.nm + 1);
    for (int m = 0; m < inner.v.nm; ++m) {
        u_first[m] = (int)u_src.size();
        for (int j = 0; j < inner.v.natoms(m); ++j) {
            u_src.push_back(m * inner.v.ma + j);
            u_lab.push_back(inner.v.q[(size_t)m * inner.v.ma + j]);
        }
    }
    u_first[inner.v.nm] = (int)u_src.size();
    const int NU = (int)u_src.size();
    const int nmo = outer.v.nm;
    if (NU == 0 || nmo == 0) return KFB_OK;
    // inner atoms sorted by label (runs lab_start), outer atoms by (label, molecule)
    std::vector<int> labs(u_lab);
    std::sort(labs.begin(), labs.end());
    labs.erase(std::unique(labs.begin(), labs.end()), labs.end());
    const int nlab = (int)labs.size();
    std::vector<int> u_sorted(NU);
    std::iota(u_sorted.begin(), u_sorted.end(), 0);
    std::stable_sort(u_sorted.begin(), u_sorted.end(),
                     [&](int a, int b) { return u_lab[a] < u_lab[b]; });
    std::vector<int> lab_start(nlab + 1, 0), in_rows(NU);
    for (int l = 0, u = 0; l < nlab; ++l) {
        lab_start[l] = u;
        while (u < NU && u_lab[u_sorted[u]] == labs[l]) ++u;
        lab_start[l + 1] = u;
    }
    for (int su = 0; su < NU; ++su) in_rows[su] = u_src[u_sorted[su]];
    std::vector<int> out_rows;
    std::vector<int2> orng((size_t)nmo * nlab);
    std::vector<int> out_lab_start(nlab + 1);
    int ns_max = 0;
    for (int l = 0; l < nlab; ++l) {
        out_lab_start[l] = (int)out_rows.size();
        for (int o = 0; o < nmo; ++o) {
            const int start = (int)out_rows.size();
            for (int i = 0; i < outer.v.natoms(o); ++i)
                if (outer.v.q[(size_t)o * outer.v.ma + i] == labs[l])
                    out_rows.push_back(o * outer.v.ma + i);
            const int cnt = (int)out_rows.size() - start;
            orng[(size_t)o * nlab + l] = make_int2(start, cnt);
            ns_max = std::max(ns_max, cnt);
        }
    }
    out_lab_start[nlab] = (int)out_rows.size();
    const int NO = (int)out_rows.size();
    // slice width of the staged outer rows: wide (fewer barriers) while the
    // block stays small enough for several blocks per SM
    int jv_lg = 8;   // 256 columns
    auto jv_bytes = [&](int lg) { return ((size_t)ns_max * (JV_U + (1 << lg)) + JV_U) * sizeof(T); };
    while (jv_lg > 6 && jv_bytes(jv_lg) > 72 * 1024) --jv_lg;
    const size_t jv_smem = jv_bytes(jv_lg);
    if (jv_smem > 200 * 1024)
        return set_error(KFB_ERR_INVALID_ARG, "%d atoms of one element in a molecule: too many "
                         "for the Jacobian kernel", ns_max);
    if (jv_smem > 48 * 1024) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(jac_v_kernel<T, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)jv_smem));
        KFB_CUDA_TRY(cudaFuncSetAttribute(jac_v_kernel<T, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)jv_smem));
    }
    // tiles of up to JV_U sorted inner atoms within one label
    std::vector<int4> tiles;
    for (int l = 0; l < nlab; ++l)
        for (int u0 = lab_start[l]; u0 < lab_start[l + 1]; u0 += JV_U)
            tiles.push_back(make_int4(l, u0, std::min(u0 + JV_U, lab_start[l + 1]), 0));
    if (tiles.size() > 65535)
        return set_error(KFB_ERR_INVALID_ARG, "%d inner atoms: too many for one Jacobian call", NU);
    // gathered rows, norms and max |x|
    DevBuf d_inrows, d_outrows, d_orng, d_usorted, d_tiles, amax, xi_s, ni_s, xo_s, no_s;
    KFB_TRY(upload(d_inrows, in_rows, s));
    KFB_TRY(upload(d_outrows, out_rows, s));
    KFB_TRY(upload(d_orng, orng, s));
    KFB_TRY(upload(d_usorted, u_sorted, s));
    KFB_TRY(upload(d_tiles, tiles, s));
    KFB_TRY(amax.alloc(2 * sizeof(float), s));
    KFB_TRY(zero(amax.ptr, 2 * sizeof(float), s));
    KFB_TRY(xi_s.alloc((size_t)NU * rep * sizeof(T), s));
    KFB_TRY(ni_s.alloc((size_t)NU * sizeof(T), s));
    KFB_TRY(xo_s.alloc(((size_t)NO * rep + 1) * sizeof(T), s));
    KFB_TRY(no_s.alloc(((size_t)NO + 1) * sizeof(T), s));
    {
        TraceScope tr("jacobian:gather", s);
        gather_rows_norm_kernel<T><<<NU, 256, 0, s>>>(static_cast<const T *>(inner.x),
                                                      d_inrows.as<int>(), NU, rep, xi_s.as<T>(),
                                                      ni_s.as<T>(), amax.as<float>());
        KFB_CUDA_TRY(cudaGetLastError());
        if (NO > 0) {
            gather_rows_norm_kernel<T><<<NO, 256, 0, s>>>(
                static_cast<const T *>(outer.x), d_outrows.as<int>(), NO, rep, xo_s.as<T>(),
                no_s.as<T>(), amax.as<float>() + 1);
            KFB_CUDA_TRY(cudaGetLastError());
        }
    }
    // outer molecules per chunk: the v rows of a chunk (T, or the fp16 pair)
    // stay resident for its contraction
    const size_t row_bytes = (size_t)NU * rep * (tc ? 2 * sizeof(__half) : sizeof(T));
    size_t budget = budget_bytes();
    if (!getenv("KFB_WORKSPACE_GB")) {
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) == cudaSuccess)
            budget = std::max(budget, std::min<size_t>(fr / 4, (size_t)16 << 30));
    }
    int chunk = (int)std::max<size_t>(1, budget / std::max<size_t>(row_bytes, 1));
    chunk = std::min(chunk, nmo);
    if (tc && chunk > 128) chunk -= chunk % 128;   // whole 128-row MMA tiles
    // dot products of a chunk: a row per matched outer atom (label blocks one
    // after the other), a column per sorted inner atom; only the label-diagonal
    // blocks are formed and read
    size_t d_elems = 1;
    for (int o0 = 0; o0 < nmo; o0 += chunk) {
        const int o1 = std::min(nmo, o0 + chunk);
        size_t rows = 0;
        for (int l = 0; l < nlab; ++l) {
            const int r0 = orng[(size_t)o0 * nlab + l].x;
            const int r1 = o1 < nmo ? orng[(size_t)o1 * nlab + l].x : out_lab_start[l + 1];
            rows += (size_t)(r1 - r0);
        }
        d_elems = std::max(d_elems, rows * (size_t)NU);
    }
    // tensor-core dot products (FP32 inputs): K-major split copies of both sets
    const bool tc_dots = tc && sizeof(T) == 4 && NO > 0;
    const int kpad = (rep + 15) / 16 * 16;
    float xi_scale = 1.f, xo_scale = 1.f;
    DevBuf V, vh, vl, jth, jtl, Dd, d_cinfo, xih, xil, xoh, xol;
    KFB_TRY(Dd.alloc(d_elems * sizeof(T), s));
    float jt_scale = 1.f, v_scale = 1.f;
    const int ma_in = inner.v.ma;
    const T c2 = T(-1.0 / (2.0 * sigma * sigma)), is2 = T(1.0 / (sigma * sigma));
    if (tc) {
        // inner Jacobians as K-major split rows: Jt[(m, c)][(j, k)]
        const size_t jt_elems = (size_t)inner.v.nm * 3 * ma_in * ma_in * rep;
        KFB_TRY(jth.alloc(jt_elems * sizeof(__half), s));
        KFB_TRY(jtl.alloc(jt_elems * sizeof(__half), s));
        std::vector<int> nin(inner.v.nm);
        for (int m = 0; m < inner.v.nm; ++m) nin[m] = inner.v.natoms(m);
        DevBuf d_nin;
        KFB_TRY(upload(d_nin, nin, s));
        TraceScope tr("jacobian:split_dx", s);
        KFB_TRY(transpose_split_dx<T>(static_cast<const T *>(inner.dx), inner.v.nm, ma_in, rep,
                                      d_nin.as<int>(), jth.as<__half>(), jtl.as<__half>(),
                                      &jt_scale, s));
        KFB_TRY(vh.alloc((size_t)chunk * NU * rep * sizeof(__half), s));
        KFB_TRY(vl.alloc((size_t)chunk * NU * rep * sizeof(__half), s));
        // |v| <= (sum_i w_iu) (max|x_out| + max|x_in|) <= ns_max / sigma^2 (...)
        float am[2] = {0.f, 0.f};
        KFB_CUDA_TRY(cudaMemcpyAsync(am, amax.ptr, sizeof(am), cudaMemcpyDeviceToHost, s));
        KFB_CUDA_TRY(cudaStreamSynchronize(s));
        const double bound = (double)ns_max / (sigma * sigma) * ((double)am[0] + (double)am[1]);
        auto pow2_for = [](double mx) {
            return (mx > 0.0 && std::isfinite(mx))
                       ? (float)std::ldexp(1.0, 14 - (int)std::ceil(std::log2(mx)))
                       : 1.f;
        };
        v_scale = pow2_for(bound);
        if (tc_dots) {
            xi_scale = pow2_for(am[0]);
            xo_scale = pow2_for(am[1]);
            KFB_TRY(xih.alloc((size_t)NU * kpad * sizeof(__half), s));
            KFB_TRY(xil.alloc((size_t)NU * kpad * sizeof(__half), s));
            KFB_TRY(xoh.alloc((size_t)NO * kpad * sizeof(__half), s));
            KFB_TRY(xol.alloc((size_t)NO * kpad * sizeof(__half), s));
            split_pad_rows_kernel<T><<<NU, 128, 0, s>>>(xi_s.as<T>(), rep, kpad, xi_scale,
                                                        xih.as<__half>(), xil.as<__half>());
            KFB_CUDA_TRY(cudaGetLastError());
            split_pad_rows_kernel<T><<<NO, 128, 0, s>>>(xo_s.as<T>(), rep, kpad, xo_scale,
                                                        xoh.as<__half>(), xol.as<__half>());
            KFB_CUDA_TRY(cudaGetLastError());
        }
    } else {
        KFB_TRY(V.alloc((size_t)chunk * NU * rep * sizeof(T), s));
    }
    cublasHandle_t h = nullptr;
    KFB_TRY(blas_for_stream(s, &h));
    const int ld_in = 3 * inner.v.ma;
    std::vector<long long> cinfo(2 * nlab);
    for (int o0 = 0; o0 < nmo; o0 += chunk) {
        const int nout = std::min(chunk, nmo - o0);
        const int o1 = o0 + nout;
        {
            TraceScope tr_d("jacobian:dots", s);
            int drow = 0;
            std::vector<TcProb> dprobs;
            for (int l = 0; l < nlab; ++l) {
                const int r0 = orng[(size_t)o0 * nlab + l].x;
                const int r1 = o1 < nmo ? orng[(size_t)o1 * nlab + l].x : out_lab_start[l + 1];
                const int nin = lab_start[l + 1] - lab_start[l];
                cinfo[l] = (long long)drow * NU;
                cinfo[nlab + l] = r0;
                if (r1 > r0 && nin > 0) {
                    // D[drow + i][lab_start[l] + u] = x_out[r0 + i] . x_in[lab_start[l] + u]
                    if (tc_dots) {
                        TcProb p{};
                        p.a_row0 = r0;
                        p.b_row0 = lab_start[l];
                        p.M = r1 - r0;
                        p.N = nin;
                        p.K = kpad;
                        p.row_off = drow;
                        p.col_off = lab_start[l];
                        p.alpha = 1.0 / ((double)xo_scale * (double)xi_scale);
                        dprobs.push_back(p);
                    } else {
                        const cublasStatus_t st = BlasGemm<T>::run(
                            h, CUBLAS_OP_T, CUBLAS_OP_N, nin, r1 - r0, rep,
                            xi_s.as<T>() + (size_t)lab_start[l] * rep, rep,
                            xo_s.as<T>() + (size_t)r0 * rep, rep,
                            Dd.as<T>() + (size_t)drow * NU + lab_start[l], NU);
                        if (st != CUBLAS_STATUS_SUCCESS)
                            return set_error(KFB_ERR_CUDA,
                                             "dot-product GEMM failed: cublas status %d", (int)st);
                    }
                }
                drow += r1 - r0;
            }
            if (!dprobs.empty()) {
                TcOperand A, B;
                A.hi = xoh.ptr;
                A.lo = xol.ptr;
                A.rows = NO;
                A.cols = kpad;
                B.hi = xih.ptr;
                B.lo = xil.ptr;
                B.rows = NU;
                B.cols = kpad;
                TcEpi epi;
                epi.mode = EPI_DENSE;
                epi.zf32 = reinterpret_cast<float *>(Dd.ptr);
                epi.ld = NU;
                KFB_TRY(tc_gemm_grouped(A, B, 3, false, dprobs, ElemSink(), s, epi));
            }
            KFB_TRY(upload(d_cinfo, cinfo, s));
        }
        {
            TraceScope tr_v("jacobian:v", s);
            const dim3 grid((unsigned)nout, (unsigned)tiles.size());
            if (tc)
                jac_v_kernel<T, true><<<grid, JV_THREADS, jv_smem, s>>>(
                    d_tiles.as<int4>(), d_orng.as<int2>(), nlab, o0, d_cinfo.as<long long>(),
                    xo_s.as<T>(), no_s.as<T>(), xi_s.as<T>(), ni_s.as<T>(),
                    Dd.as<T>(), d_usorted.as<int>(), NU, rep, jv_lg, c2, T(is2 * (T)v_scale),
                    nullptr, vh.as<__half>(), vl.as<__half>());
            else
                jac_v_kernel<T, false><<<grid, JV_THREADS, jv_smem, s>>>(
                    d_tiles.as<int4>(), d_orng.as<int2>(), nlab, o0, d_cinfo.as<long long>(),
                    xo_s.as<T>(), no_s.as<T>(), xi_s.as<T>(), ni_s.as<T>(),
                    Dd.as<T>(), d_usorted.as<int>(), NU, rep, jv_lg, c2, is2, V.as<T>(), nullptr,
                    nullptr);
            KFB_CUDA_TRY(cudaGetLastError());
        }
        TraceScope tr_c("jacobian:gemm", s);
        if (tc) {
            std::vector<TcProb> tprobs;
            for (int m = 0; m < inner.v.nm; ++m) {
                const int nb = inner.v.natoms(m);
                if (nb == 0) continue;
                TcProb p{};
                p.a_row0 = 0;
                p.a_k0 = u_first[m] * rep;
                p.b_row0 = m * 3 * ma_in;
                p.b_k0 = 0;
                p.M = nout;
                p.N = 3 * nb;
                p.K = nb * rep;
                p.row_off = o0;
                p.col_off = in_offs[m];
                p.diag = 0;
                p.alpha = alpha / ((double)v_scale * (double)jt_scale);
                tprobs.push_back(p);
            }
            TcOperand A, B;
            A.hi = vh.ptr;
            A.lo = vl.ptr;
            A.rows = nout;
            A.cols = (long long)NU * rep;
            B.hi = jth.ptr;
            B.lo = jtl.ptr;
            B.rows = (long long)inner.v.nm * 3 * ma_in;
            B.cols = (long long)ma_in * rep;
            // longest problems first: the persistent CTAs take tiles in list
            // order, so the ragged ends of the K loops fall in the last wave
            std::stable_sort(tprobs.begin(), tprobs.end(),
                             [](const TcProb &x, const TcProb &y) { return x.K > y.K; });
            KFB_TRY(tc_gemm_grouped(A, B, 3, false, tprobs, sink, s));
            continue;
        }
        std::vector<GemmProb> probs;
        for (int m = 0; m < inner.v.nm; ++m) {
            const int nb = inner.v.natoms(m);
            if (nb == 0) continue;
            GemmProb p{};
            p.A = V.as<T>() + (size_t)u_first[m] * rep;
            p.lda = (long long)NU * rep;
            p.transA = 0;
            p.B = static_cast<const T *>(inner.dx) + (size_t)m * inner.v.ma * rep * ld_in;
            p.ldb = ld_in;
            p.M = nout;
            p.N = 3 * nb;
            p.K = nb * rep;
            p.row_off = o0;
            p.col_off = in_offs[m];
            p.alpha = alpha;
            p.diag = 0;
            probs.push_back(p);
        }
        KFB_TRY(launch_gemm<T>(probs, sink, s));
    }
    return KFB_OK;
}

// ---------------------------------------------------------------------------
// Hessian core: H_ab blocks for the listed molecule pairs, through `sink`
// (rows offset by off1[a], columns by off2[b]).
// ---------------------------------------------------------------------------
// Atoms of a set in label-major order (label index, then molecule, then atom):
// cum[l (nm + 1) + m] = label-l atoms in molecules < m, start[l] = label-major
// index of label l's first atom, rank[m ma + i] = label-major index of atom
// (m, i) (-1: no label index), src[r] = m ma + i of label-major atom r.  The
// label-l atoms of molecules m0..m1 are the contiguous range from first(l, m0).
struct LabelMajor {
    int L = 0, nm = 0, n = 0;
    std::vector<int> cum, start, rank, src, lab;
    void build(const std::vector<int> &lidx, int nm_, int ma, int L_) {
        L = L_;
        nm = nm_;
        lab = lidx;
        cum.assign((size_t)L * (nm + 1), 0);
        for (int m = 0; m < nm; ++m) {
            for (int l = 0; l < L; ++l) cum[(size_t)l * (nm + 1) + m + 1] = cum[(size_t)l * (nm + 1) + m];
            for (int i = 0; i < ma; ++i) {
                const int l = lidx[(size_t)m * ma + i];
                if (l >= 0) ++cum[(size_t)l * (nm + 1) + m + 1];
            }
        }
        start.assign(L + 1, 0);
        for (int l = 0; l < L; ++l) start[l + 1] = start[l] + cum[(size_t)l * (nm + 1) + nm];
        n = start[L];
        rank.assign((size_t)nm * ma, -1);
        src.assign(n, 0);
        std::vector<int> within(L);
        for (int m = 0; m < nm; ++m) {
            std::fill(within.begin(), within.end(), 0);
            for (int i = 0; i < ma; ++i) {
                const int l = lidx[(size_t)m * ma + i];
                if (l < 0) continue;
                const int r = first(l, m) + within[l]++;
                rank[(size_t)m * ma + i] = r;
                src[r] = m * ma + i;
            }
        }
    }
    int first(int l, int m) const { return start[l] + cum[(size_t)l * (nm + 1) + m]; }
    int count(int l, int m0, int m1) const {
        return cum[(size_t)l * (nm + 1) + m1 + 1] - cum[(size_t)l * (nm + 1) + m0];
    }
};

// dst rows r = src rows srcrow[r] of an fp16 pair (rep entries per row)
__global__ void gather_rows_kernel(const __half *__restrict__ shi, const __half *__restrict__ slo,
                                   const int *__restrict__ srcrow, int rep,
                                   __half *__restrict__ dhi, __half *__restrict__ dlo) {
    const size_t r = blockIdx.x, sr = (size_t)srcrow[r];
    for (int k = threadIdx.x; k < rep; k += blockDim.x) {
        dhi[r * rep + k] = shi[sr * rep + k];
        dlo[r * rep + k] = slo[sr * rep + k];
    }
}

// Label-major copy (lm.n rows) of a split row array in atom order.
kfb_status label_major_rows(const LabelMajor &lm, const DevBuf &hi, const DevBuf &lo, int rep,
                            DevBuf &dhi, DevBuf &dlo, cudaStream_t s) {
    if (lm.n == 0) return KFB_OK;
    DevBuf d_src;
    KFB_TRY(upload(d_src, lm.src, s));
    KFB_TRY(dhi.alloc((size_t)lm.n * rep * sizeof(__half), s));
    KFB_TRY(dlo.alloc((size_t)lm.n * rep * sizeof(__half), s));
    gather_rows_kernel<<<(unsigned)lm.n, 128, 0, s>>>(hi.as<__half>(), lo.as<__half>(),
                                                     d_src.as<int>(), rep, dhi.as<__half>(),
                                                     dlo.as<__half>());
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

// Projection problems of a batch, one per label: rows = the label-l atoms of
// molecules r0..r1 of set R (its label-major rows), columns = cw rows per
// label-l atom of molecules c0..c1 of set C (label-major blocks of cw rows);
// problem rows stacked from 0.  rowmap[(m - r0) mar + i] = output row of atom
// (m, i), colmap[(m - c0) mac + j] = first output column of atom (m, j) (-1:
// no problem).  Returns the output row length (widest problem, rounded up to 8).
long long label_problems(const LabelMajor &R, int r0, int r1, int mar, const LabelMajor &C,
                         int c0, int c1, int mac, int cw, int K, double alpha,
                         std::vector<TcProb> &probs, std::vector<int> &rowmap,
                         std::vector<int> &colmap) {
    probs.clear();
    std::vector<int> rowbase(R.L, -1);
    long long ld = 0;
    int rb = 0;
    for (int l = 0; l < R.L; ++l) {
        const int M = R.count(l, r0, r1), Nn = C.count(l, c0, c1);
        if (M == 0 || Nn == 0) continue;
        TcProb p{};
        p.a_row0 = R.first(l, r0);
        p.b_row0 = C.first(l, c0) * cw;
        p.M = M;
        p.N = Nn * cw;
        p.K = K;
        p.row_off = rb;
        p.alpha = alpha;
        probs.push_back(p);
        rowbase[l] = rb;
        rb += M;
        ld = std::max(ld, (long long)p.N);
    }
    rowmap.assign((size_t)(r1 - r0 + 1) * mar, -1);
    for (int m = r0; m <= r1; ++m)
        for (int i = 0; i < mar; ++i) {
            const size_t a = (size_t)m * mar + i;
            const int l = R.lab[a];
            if (l >= 0 && rowbase[l] >= 0)
                rowmap[(size_t)(m - r0) * mar + i] = rowbase[l] + R.rank[a] - R.first(l, r0);
        }
    colmap.assign((size_t)(c1 - c0 + 1) * mac, -1);
    for (int m = c0; m <= c1; ++m)
        for (int j = 0; j < mac; ++j) {
            const size_t a = (size_t)m * mac + j;
            const int l = C.lab[a];
            if (l >= 0 && rowbase[l] >= 0)
                colmap[(size_t)(m - c0) * mac + j] = (C.rank[a] - C.first(l, c0)) * cw;
        }
    return (ld + 7) / 8 * 8;
}

// Y of a batch by the tensor cores: a GEMM problem per molecule b of the
// batch (pairs with that b, in b order, as columns (q, i)), see jk_split_kernel.
kfb_status hess_y_gemm(const HessPair *pairs, int np, int ma1, int ma2, int rep, int kj,
                       const float *W, const DevBuf &jkh, const DevBuf &jkl, float jk_scale,
                       float w_scale, float y_scale, DevBuf &wsh, DevBuf &wsl, DevBuf &d_ymap,
                       DevBuf &d_border, long long jk_rows, __half *yhi, __half *ylo,
                       cudaStream_t s) {
    const int ld2 = 3 * ma2;
    std::vector<int> border(np);
    for (int p = 0; p < np; ++p) border[p] = p;
    std::stable_sort(border.begin(), border.end(),
                     [&](int x, int y) { return pairs[x].b < pairs[y].b; });
    std::vector<int2> ymap((size_t)np * ma1);
    std::vector<TcProb> probs;
    for (int q = 0; q < np;) {
        const HessPair &pr = pairs[border[q]];
        int q1 = q;
        for (; q1 < np && pairs[border[q1]].b == pr.b; ++q1) {
            const int p = border[q1];
            for (int i = 0; i < ma1; ++i)
                ymap[(size_t)q1 * ma1 + i] = make_int2(i < pairs[p].na ? p : -1, i);
        }
        TcProb pb{};
        pb.a_row0 = (int)((long long)pr.b * ld2 * rep);
        pb.b_row0 = q * ma1;
        pb.M = 3 * pr.nb * rep;
        pb.N = (q1 - q) * ma1;
        pb.K = kj;
        pb.alpha = (double)y_scale / ((double)jk_scale * (double)w_scale);
        probs.push_back(pb);
        q = q1;
    }
    KFB_CUDA_TRY(cudaMemcpyAsync(d_border.ptr, border.data(), (size_t)np * sizeof(int),
                                 cudaMemcpyHostToDevice, s));
    KFB_CUDA_TRY(cudaMemcpyAsync(d_ymap.ptr, ymap.data(), ymap.size() * sizeof(int2),
                                 cudaMemcpyHostToDevice, s));
    const int nrows = np * ma1;
    const long long nthr = (long long)nrows * (kj / 8);
    w_split_kernel<<<(unsigned)((nthr + 255) / 256), 256, 0, s>>>(
        W, d_border.as<int>(), nrows, ma1, ma2, kj, w_scale, wsh.as<__half>(), wsl.as<__half>());
    KFB_CUDA_TRY(cudaGetLastError());
    TcOperand A, B;
    A.hi = jkh.ptr;
    A.lo = jkl.ptr;
    A.rows = jk_rows;
    A.cols = kj;
    B.hi = wsh.ptr;
    B.lo = wsl.ptr;
    B.rows = nrows;
    B.cols = kj;
    TcEpi epi;
    epi.mode = EPI_YSPLIT;
    epi.ymap = d_ymap.as<int2>();
    epi.yhi = yhi;
    epi.ylo = ylo;
    epi.y_rep = rep;
    epi.y_ma1 = ma1;
    epi.y_ld2 = ld2;
    return tc_gemm_grouped(A, B, 3, false, probs, ElemSink(), s, epi);
}

template <class T>
kfb_status hessian_core(const DerivSet &s1, const DerivSet &s2, int rep, double sigma,
                        bool symmetric, bool tc, ElemSink sink, cudaStream_t s) {
    std::vector<int> off1, off2;
    deriv_offsets(s1.v, off1);
    deriv_offsets(s2.v, off2);
    // pairs ordered by b: the Y kernels stream molecule b's Jacobian, which
    // then stays in L2 across the consecutive pairs that share it
    std::vector<HessPair> pairs;
    for (int b = 0; b < s2.v.nm; ++b) {
        const int nb = s2.v.natoms(b);
        if (nb == 0) continue;
        for (int a = 0; a < (symmetric ? b + 1 : s1.v.nm); ++a) {
            const int na = s1.v.natoms(a);
            if (na == 0) continue;
            pairs.push_back(HessPair{a, b, na, nb});
        }
    }
    if (pairs.empty()) return KFB_OK;
    const int ma1 = s1.v.ma, ma2 = s2.v.ma, ld1 = 3 * ma1, ld2 = 3 * ma2;
    // scratch per pair: W, Tt, and Y (T) or its fp16 pair (tensor cores)
    const size_t per_pair = (size_t)ma1 * ma2 * (1 + ld2) * sizeof(T) +
                            (size_t)ma1 * rep * ld2 * (tc ? 2 * sizeof(__half) : sizeof(T));
    int batch = (int)std::max<size_t>(1, budget_bytes() / per_pair);
    batch = std::min<int>(batch, (int)pairs.size());
    batch = std::min(batch, 65535);
    DevBuf W, Tt, Y, dpairs;
    KFB_TRY(W.alloc((size_t)batch * ma1 * ma2 * sizeof(T), s));
    KFB_TRY(Tt.alloc((size_t)batch * ma1 * ma2 * ld2 * sizeof(T), s));
    if (!tc) KFB_TRY(Y.alloc((size_t)batch * ma1 * rep * ld2 * sizeof(T), s));
    KFB_TRY(dpairs.alloc((size_t)batch * sizeof(HessPair), s));
    std::vector<int> perm1, lab1, perm2, lab2;
    label_order(s1.v, perm1, lab1);
    label_order(s2.v, perm2, lab2);
    DevBuf d_perm1, d_lab1, d_perm2, d_lab2;
    KFB_TRY(upload(d_perm1, perm1, s));
    KFB_TRY(upload(d_lab1, lab1, s));
    KFB_TRY(upload(d_perm2, perm2, s));
    KFB_TRY(upload(d_lab2, lab2, s));
    DevBuf jth, jtl, yth, ytl, yamax;
    float jt_scale = 1.f;
    if (tc) {
        // set-1 Jacobians as K-major split rows Jt[(a, c)][(i, k)]
        const size_t jt_elems = (size_t)s1.v.nm * ld1 * ma1 * rep;
        KFB_TRY(jth.alloc(jt_elems * sizeof(__half), s));
        KFB_TRY(jtl.alloc(jt_elems * sizeof(__half), s));
        std::vector<int> n1(s1.v.nm);
        for (int m = 0; m < s1.v.nm; ++m) n1[m] = s1.v.natoms(m);
        DevBuf d_n1;
        KFB_TRY(upload(d_n1, n1, s));
        KFB_TRY(transpose_split_dx<T>(static_cast<const T *>(s1.dx), s1.v.nm, ma1, rep,
                                      d_n1.as<int>(), jth.as<__half>(), jtl.as<__half>(),
                                      &jt_scale, s));
        KFB_TRY(yamax.alloc(sizeof(float), s));
        KFB_TRY(yth.alloc((size_t)batch * ld2 * ma1 * rep * sizeof(__half), s));
        KFB_TRY(ytl.alloc((size_t)batch * ld2 * ma1 * rep * sizeof(__half), s));
    }
    const T c2 = T(-1.0 / (2.0 * sigma * sigma)), is2 = T(1.0 / (sigma * sigma));
    const T is4 = is2 * is2;
    // Kernel 1 in GEMM form (tensor cores, FP32 inputs): P = (X1 - mu) Jr^T per
    // batch of molecules b, with per-label centres mu of set 1.  Needs the P
    // columns of one molecule b for every set-1 atom within half the workspace
    // and at most 16 labels; otherwise kernel 1 forms J_j^T d_ij itself.
    const long long Mrows = (long long)s1.v.nm * ma1, bcols = (long long)ma2 * ld2;
    // With the GEMM form the rank term of Y moves to hess_rank_kernel (hrank):
    // Q = (X2 - mu) Jr1^T per batch, set-1 Jacobian rows (a, i, c') as columns.
    const long long Mq = (long long)s1.v.nm * ma1 * ld1;
    bool pform = false, hrank = false;
    int bcap = 0;
    float xs_scale = 1.f, jr_scale = 1.f, jr1_scale = 1.f;
    DevBuf d_l1, d_l2, d_sums, d_invc, d_amx, xh1, xl1, jrh, jrl, d_pb, d_jbm, d_P, d_nat2,
        d_n1, xh2, xl2, d_n2, d_G, jr1h, jr1l, d_pb1, d_Q, d_off1, d_off2, d_nat1;
    // the P and Q projections pair same-label atoms only: their operands in
    // label-major order (x1L/x2L: centred descriptor rows, jrh/jr1h: Jacobian
    // rows), one GEMM problem per label, and per-batch maps from atoms to rows
    // and columns of P and Q
    LabelMajor lm1, lm2;
    DevBuf x1Lh, x1Ll, x2Lh, x2Ll, d_rank1, d_rank2, d_prow, d_pcol, d_qrow, d_qcol;
    float xs2_scale = 1.f;
    // Y on the tensor cores (rank term outside Y): set 2's Jacobian as rows
    // (b, c, k) with kj atom columns, resident for the call
    bool ygemm = false;
    int kj = 0;
    float w_scale = 1.f;
    DevBuf jkh, jkl, wsh, wsl, d_ymap, d_border;
    if constexpr (std::is_same<T, float>::value) {
        const std::vector<int> labs1 = collect_labels(s1.v, nullptr);
        const long long pbytes = Mrows * bcols * (long long)sizeof(float);
        pform = tc && !labs1.empty() && labs1.size() <= 16 &&
                pbytes <= (long long)(budget_bytes() / 2) && Mrows < INT_MAX &&
                (long long)s2.v.nm * bcols < INT_MAX;
        const long long qbytes = Mq * ma2 * (long long)sizeof(float);
        hrank = pform && ma1 <= HR_MAXA && ma2 <= HR_MAXA && Mq < INT_MAX &&
                pbytes + qbytes <= (long long)(budget_bytes() / 2);
        if (hrank && !symmetric) {
            // an asymmetric call also keeps set 1's split Jacobian rows and PB1
            // resident (outside the batch budget): take the rank kernel only
            // when they fit in free memory next to a full workspace, else keep
            // the rank term inside Y
            const long long r1bytes = Mq * (long long)rep * 2 * (long long)sizeof(__half) +
                                      Mq * (long long)sizeof(float);
            size_t free_b = 0, total_b = 0;
            KFB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
            hrank = r1bytes + (long long)budget_bytes() <= (long long)free_b;
        }
        note_path(!pform ? "hessian:cuda-core-t" : (hrank ? "hessian:rank-kernel"
                                                           : "hessian:rank-in-y"));
        if (pform) {
            TraceScope tr_p("hessian:p-setup", s);
            const int L = (int)labs1.size();
            auto lab_index = [&](int q) {
                const auto it = std::lower_bound(labs1.begin(), labs1.end(), q);
                return (it != labs1.end() && *it == q) ? (int)(it - labs1.begin()) : -1;
            };
            std::vector<int> l1((size_t)Mrows, -1), l2((size_t)s2.v.nm * ma2, -1), nat2(s2.v.nm);
            std::vector<double> cnt(L, 0.0), invc(L, 0.0);
            for (int m = 0; m < s1.v.nm; ++m)
                for (int i = 0; i < s1.v.natoms(m); ++i) {
                    const int l = lab_index(s1.v.q[(size_t)m * ma1 + i]);
                    l1[(size_t)m * ma1 + i] = l;
                    if (l >= 0) cnt[l] += 1.0;
                }
            for (int m = 0; m < s2.v.nm; ++m) {
                nat2[m] = s2.v.natoms(m);
                for (int j = 0; j < nat2[m]; ++j)
                    l2[(size_t)m * ma2 + j] = lab_index(s2.v.q[(size_t)m * ma2 + j]);
            }
            for (int l = 0; l < L; ++l) invc[l] = cnt[l] > 0.0 ? 1.0 / cnt[l] : 0.0;
            lm1.build(l1, s1.v.nm, ma1, L);
            lm2.build(l2, s2.v.nm, ma2, L);
            KFB_TRY(upload(d_l1, l1, s));
            KFB_TRY(upload(d_l2, l2, s));
            KFB_TRY(upload(d_invc, invc, s));
            KFB_TRY(upload(d_nat2, nat2, s));
            KFB_TRY(d_sums.alloc((size_t)L * rep * sizeof(double), s));
            KFB_TRY(zero(d_sums.ptr, (size_t)L * rep * sizeof(double), s));
            const float *x1f = static_cast<const float *>(s1.x);
            const float *x2f = static_cast<const float *>(s2.x);
            const float *dx2f = static_cast<const float *>(s2.dx);
            label_sums_kernel<float><<<dim3((unsigned)((rep + 31) / 32), 16), 256,
                                       (size_t)L * 256 * sizeof(double), s>>>(
                x1f, d_l1.as<int>(), (int)Mrows, rep, L, d_sums.as<double>());
            KFB_CUDA_TRY(cudaGetLastError());
            KFB_TRY(d_amx.alloc(sizeof(float), s));
            KFB_TRY(zero(d_amx.ptr, sizeof(float), s));
            const unsigned ab = (unsigned)std::min<long long>((Mrows * rep + 255) / 256, 148LL * 8);
            centred_absmax_kernel<float><<<ab, 256, 0, s>>>(x1f, d_l1.as<int>(), (int)Mrows, rep,
                                                            d_sums.as<double>(),
                                                            d_invc.as<double>(), d_amx.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            KFB_TRY(pow2_from_device(d_amx.as<float>(), s, &xs_scale));
            KFB_TRY(xh1.alloc((size_t)Mrows * rep * sizeof(__half), s));
            KFB_TRY(xl1.alloc((size_t)Mrows * rep * sizeof(__half), s));
            KFB_TRY(d_n1.alloc((size_t)Mrows * sizeof(float), s));
            centred_split_kernel<float><<<(unsigned)Mrows, 256, 0, s>>>(
                x1f, d_l1.as<int>(), rep, d_sums.as<double>(), d_invc.as<double>(), xs_scale,
                xh1.as<__half>(), xl1.as<__half>(), d_n1.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            // set 2, centred on the set-1 means of its labels (the same rows for
            // a symmetric call)
            const long long M2rows = (long long)s2.v.nm * ma2;
            xs2_scale = xs_scale;
            if (!symmetric) {
                KFB_TRY(zero(d_amx.ptr, sizeof(float), s));
                const unsigned ab2 =
                    (unsigned)std::min<long long>((M2rows * rep + 255) / 256, 148LL * 8);
                centred_absmax_kernel<float><<<ab2, 256, 0, s>>>(
                    x2f, d_l2.as<int>(), (int)M2rows, rep, d_sums.as<double>(),
                    d_invc.as<double>(), d_amx.as<float>());
                KFB_CUDA_TRY(cudaGetLastError());
                KFB_TRY(pow2_from_device(d_amx.as<float>(), s, &xs2_scale));
                KFB_TRY(xh2.alloc((size_t)M2rows * rep * sizeof(__half), s));
                KFB_TRY(xl2.alloc((size_t)M2rows * rep * sizeof(__half), s));
                KFB_TRY(d_n2.alloc((size_t)M2rows * sizeof(float), s));
                centred_split_kernel<float><<<(unsigned)M2rows, 256, 0, s>>>(
                    x2f, d_l2.as<int>(), rep, d_sums.as<double>(), d_invc.as<double>(),
                    xs2_scale, xh2.as<__half>(), xl2.as<__half>(), d_n2.as<float>());
                KFB_CUDA_TRY(cudaGetLastError());
            }
            KFB_TRY(label_major_rows(lm1, xh1, xl1, rep, x1Lh, x1Ll, s));
            if (!symmetric) KFB_TRY(label_major_rows(lm2, xh2, xl2, rep, x2Lh, x2Ll, s));
            // set-2 Jacobian rows, label-major blocks of ld2 rows per atom
            KFB_TRY(upload(d_rank2, lm2.rank, s));
            const size_t jr_elems = std::max<size_t>(1, (size_t)lm2.n * ld2 * rep);
            KFB_TRY(jrh.alloc(jr_elems * sizeof(__half), s));
            KFB_TRY(jrl.alloc(jr_elems * sizeof(__half), s));
            KFB_TRY(transpose_split_dx_rows<float>(dx2f, s2.v.nm, ma2, rep, d_nat2.as<int>(),
                                                   jrh.as<__half>(), jrl.as<__half>(),
                                                   &jr_scale, s, d_rank2.as<int>()));
            KFB_TRY(d_pb.alloc((size_t)s2.v.nm * bcols * sizeof(float), s));
            pb_kernel<float><<<(unsigned)(s2.v.nm * ma2), 128, 0, s>>>(
                x2f, dx2f, d_l2.as<int>(), ma2, rep, d_sums.as<double>(), d_invc.as<double>(),
                d_pb.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            KFB_TRY(d_jbm.alloc((size_t)s2.v.nm * sizeof(float), s));
            KFB_TRY(zero(d_jbm.ptr, (size_t)s2.v.nm * sizeof(float), s));
            jmax_per_mol_kernel<float><<<dim3((unsigned)s2.v.nm, 32), 256, 0, s>>>(
                dx2f, ma2, rep, d_nat2.as<int>(), d_jbm.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            if (hrank) {
                // set-1 Jacobian rows and PB1 (the set-2 ones for a symmetric call)
                jr1_scale = jr_scale;
                if (!symmetric) {
                    const float *dx1f = static_cast<const float *>(s1.dx);
                    std::vector<int> nat1(s1.v.nm);
                    for (int m = 0; m < s1.v.nm; ++m) nat1[m] = s1.v.natoms(m);
                    KFB_TRY(upload(d_nat1, nat1, s));
                    KFB_TRY(upload(d_rank1, lm1.rank, s));
                    const size_t jr1_elems = std::max<size_t>(1, (size_t)lm1.n * ld1 * rep);
                    KFB_TRY(jr1h.alloc(jr1_elems * sizeof(__half), s));
                    KFB_TRY(jr1l.alloc(jr1_elems * sizeof(__half), s));
                    KFB_TRY(transpose_split_dx_rows<float>(
                        dx1f, s1.v.nm, ma1, rep, d_nat1.as<int>(), jr1h.as<__half>(),
                        jr1l.as<__half>(), &jr1_scale, s, d_rank1.as<int>()));
                    KFB_TRY(d_pb1.alloc((size_t)Mq * sizeof(float), s));
                    pb_kernel<float><<<(unsigned)Mrows, 128, 0, s>>>(
                        x1f, dx1f, d_l1.as<int>(), ma1, rep, d_sums.as<double>(),
                        d_invc.as<double>(), d_pb1.as<float>());
                    KFB_CUDA_TRY(cudaGetLastError());
                }
                KFB_TRY(upload(d_off1, off1, s));
                KFB_TRY(upload(d_off2, off2, s));
            }
            bcap = (int)std::max<long long>(
                1, (long long)(budget_bytes() / 2) / (pbytes + (hrank ? qbytes : 0)));
            int span_max = 1;
            for (size_t q0 = 0; q0 < pairs.size(); q0 += batch) {
                const size_t q1 = std::min(pairs.size(), q0 + batch) - 1;
                span_max = std::max(span_max, pairs[q1].b - pairs[q0].b + 1);
            }
            bcap = std::min(bcap, span_max);
            // label blocks of P and Q: at most the batch's rows, row length
            // rounded up to 8
            KFB_TRY(d_P.alloc((size_t)Mrows * ((size_t)bcap * bcols + 8) * sizeof(float), s));
            KFB_TRY(d_G.alloc((size_t)bcap * Mrows * ma2 * sizeof(float), s));
            if (hrank) KFB_TRY(d_Q.alloc((size_t)bcap * ma2 * (Mq + 8) * sizeof(float), s));
            KFB_TRY(d_prow.alloc((size_t)Mrows * sizeof(int), s));
            KFB_TRY(d_pcol.alloc((size_t)s2.v.nm * ma2 * sizeof(int), s));
            if (hrank) {
                KFB_TRY(d_qrow.alloc((size_t)s2.v.nm * ma2 * sizeof(int), s));
                KFB_TRY(d_qcol.alloc((size_t)Mrows * sizeof(int), s));
            }
            if (hrank) {
                kj = (ma2 + 15) / 16 * 16;
                const long long jk_rows = (long long)s2.v.nm * ld2 * rep;
                const long long jk_bytes = jk_rows * kj * 2 * (long long)sizeof(__half);
                size_t free_b = 0, total_b = 0;
                KFB_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
                const char *ye = std::getenv("KFB_HESSIAN_Y");
                ygemm = !(ye && std::string(ye) == "cuda-core") && rep % 8 == 0 &&
                        jk_rows < INT_MAX &&
                        (long long)batch * ma1 < INT_MAX &&
                        jk_bytes + (long long)budget_bytes() <= (long long)free_b;
            }
            if (ygemm) {
                TraceScope tr_j("hessian:jk-split", s);
                const size_t jk_elems = (size_t)s2.v.nm * ld2 * rep * kj;
                KFB_TRY(jkh.alloc(jk_elems * sizeof(__half), s));
                KFB_TRY(jkl.alloc(jk_elems * sizeof(__half), s));
                const size_t jsm = (size_t)8 * (ld2 + 1) * sizeof(float);
                if (jsm > 48 * 1024)
                    KFB_CUDA_TRY(cudaFuncSetAttribute(jk_split_kernel<float>,
                                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                      (int)jsm));
                jk_split_kernel<float><<<dim3((unsigned)rep, (unsigned)s2.v.nm), 128, jsm, s>>>(
                    static_cast<const float *>(s2.dx), ma2, rep, kj, d_nat2.as<int>(), jr_scale,
                    jkh.as<__half>(), jkl.as<__half>());
                KFB_CUDA_TRY(cudaGetLastError());
                KFB_TRY(wsh.alloc((size_t)batch * ma1 * kj * sizeof(__half), s));
                KFB_TRY(wsl.alloc((size_t)batch * ma1 * kj * sizeof(__half), s));
                KFB_TRY(d_ymap.alloc((size_t)batch * ma1 * sizeof(int2), s));
                KFB_TRY(d_border.alloc((size_t)batch * sizeof(int), s));
                // 0 < w <= 1 / sigma^2: a fixed power of two brings it under 2^14
                w_scale = std::exp2(std::floor(std::log2(16384.0 * sigma * sigma)));
            }
            note_path(ygemm ? "hessian:y-gemm" : "hessian:y-cuda-core");
        }
    } else {
        note_path("hessian:cuda-core-t");
    }
    const size_t smem_p = hess_t_p_smem(ma1, ma2);
    for (size_t p0 = 0, npz = 0; p0 < pairs.size(); p0 += npz) {
        int np = (int)std::min<size_t>(batch, pairs.size() - p0);
        if (pform)  // the batch's molecules b fit the P buffer
            while (np > 1 && pairs[p0 + np - 1].b - pairs[p0].b + 1 > bcap) --np;
        npz = (size_t)np;
        const int bmin = pairs[p0].b, bmax = pairs[p0 + np - 1].b;
        // tensor-core contraction: the batch's pairs by (a, b), so that pairs
        // (a, b), (a, b + 1) of whole molecules b can share one GEMM problem
        // (their rows of Y and their output columns are adjacent)
        if (tc)
            std::stable_sort(pairs.begin() + p0, pairs.begin() + p0 + np,
                             [](const HessPair &x, const HessPair &y) {
                                 return x.a != y.a ? x.a < y.a : x.b < y.b;
                             });
        KFB_CUDA_TRY(cudaMemcpyAsync(dpairs.ptr, pairs.data() + p0, np * sizeof(HessPair),
                                     cudaMemcpyHostToDevice, s));
        const T *x1p = static_cast<const T *>(s1.x), *x2p = static_cast<const T *>(s2.x);
        const T *dx2p = static_cast<const T *>(s2.dx);
        auto tr_t = std::make_unique<TraceScope>("hessian:t", s);
        // with tensor cores kernel 1 also bounds |Y| for the power-of-two
        // scale of the fp16 split that kernel 2 writes
        if (tc) KFB_TRY(zero(yamax.ptr, sizeof(float), s));
        if constexpr (std::is_same<T, float>::value) {
            if (pform) {
                // rows of the batch's molecules a only (pairs sorted by a):
                // P and G keep their global row index
                const int amin = pairs[p0].a, amax = pairs[p0 + np - 1].a;
                const int arow0 = amin * ma1;
                const int arows = (amax + 1) * ma1 - arow0;
                std::vector<TcProb> pps;
                std::vector<int> prow, pcol;
                const long long ldp = label_problems(
                    lm1, amin, amax, ma1, lm2, bmin, bmax, ma2, ld2, rep,
                    1.0 / ((double)xs_scale * (double)jr_scale), pps, prow, pcol);
                KFB_CUDA_TRY(cudaMemcpyAsync(d_prow.ptr, prow.data(), prow.size() * sizeof(int),
                                             cudaMemcpyHostToDevice, s));
                KFB_CUDA_TRY(cudaMemcpyAsync(d_pcol.ptr, pcol.data(), pcol.size() * sizeof(int),
                                             cudaMemcpyHostToDevice, s));
                TcOperand A, B;
                A.hi = x1Lh.ptr;
                A.lo = x1Ll.ptr;
                A.rows = lm1.n;
                A.cols = rep;
                B.hi = jrh.ptr;
                B.lo = jrl.ptr;
                B.rows = (long long)lm2.n * ld2;
                B.cols = rep;
                TcEpi epi;
                epi.mode = EPI_DENSE;
                epi.zf32 = d_P.as<float>();
                epi.ld = ldp;
                KFB_TRY(tc_gemm_grouped(A, B, 3, false, pps, ElemSink(), s, epi));
                TcOperand A1;  // centred set-1 rows in atom order
                A1.hi = xh1.ptr;
                A1.lo = xl1.ptr;
                A1.rows = Mrows;
                A1.cols = rep;
                // centred dot products of the batch's atom pairs
                TcProb pg{};
                pg.a_row0 = arow0;
                pg.row_off = arow0;
                pg.b_row0 = bmin * ma2;
                pg.M = arows;
                pg.N = (bmax - bmin + 1) * ma2;
                pg.K = rep;
                pg.alpha = 1.0 / ((double)xs_scale * (double)xs2_scale);
                TcOperand B2;
                B2.hi = symmetric ? xh1.ptr : xh2.ptr;
                B2.lo = symmetric ? xl1.ptr : xl2.ptr;
                B2.rows = (long long)s2.v.nm * ma2;
                B2.cols = rep;
                TcEpi eg;
                eg.mode = EPI_DENSE;
                eg.zf32 = d_G.as<float>();
                eg.ld = pg.N;
                KFB_TRY(tc_gemm_grouped(A1, B2, 3, false, {pg}, ElemSink(), s, eg));
                // the Y GEMM reads every weight: those of other-label pairs are 0
                if (ygemm) KFB_TRY(zero(W.ptr, (size_t)np * ma1 * ma2 * sizeof(float), s));
                hess_t_p_kernel<<<np, 256, smem_p, s>>>(
                    dpairs.as<HessPair>(), d_G.as<float>(), pg.N, d_n1.as<float>(),
                    symmetric ? d_n1.as<float>() : d_n2.as<float>(), d_perm1.as<int>(),
                    d_lab1.as<int>(), d_perm2.as<int>(), d_lab2.as<int>(), ma1, ma2, c2, is2, is4,
                    d_P.as<float>(), ldp, d_prow.as<int>(), d_pcol.as<int>(), amin, bmin,
                    d_pb.as<float>(), d_jbm.as<float>(),
                    hrank ? 0 : 1, W.as<T>(), Tt.as<T>(), yamax.as<float>());
                KFB_CUDA_TRY(cudaGetLastError());
            }
        }
        if (!pform)
            KFB_TRY(launch_hess_t<T>(dpairs.as<HessPair>(), np, x1p, x2p, dx2p,
                                     d_perm1.as<int>(), d_lab1.as<int>(), d_perm2.as<int>(),
                                     d_lab2.as<int>(), ma1, ma2, rep, c2, is2, is4, W.as<T>(),
                                     Tt.as<T>(), tc ? yamax.as<float>() : nullptr, s));
        tr_t.reset();
        auto tr_y = std::make_unique<TraceScope>("hessian:y", s);
        float y_scale = 1.f;
        if (tc) {
            KFB_TRY(pow2_from_device(yamax.as<float>(), s, &y_scale));
            if (ygemm)
                KFB_TRY(hess_y_gemm(pairs.data() + p0, np, ma1, ma2, rep, kj, W.as<float>(),
                                    jkh, jkl, jr_scale, w_scale, y_scale, wsh, wsl, d_ymap,
                                    d_border, (long long)s2.v.nm * ld2 * rep, yth.as<__half>(),
                                    ytl.as<__half>(), s));
            else if (hrank)
                KFB_TRY((launch_hess_y<T, 3>(dpairs.as<HessPair>(), np, x1p, x2p, dx2p,
                                             d_perm1.as<int>(), d_lab1.as<int>(),
                                             d_perm2.as<int>(), d_lab2.as<int>(), ma1, ma2, rep,
                                             W.as<T>(), Tt.as<T>(), y_scale, yth.as<__half>(),
                                             ytl.as<__half>(), nullptr, s)));
            else
                KFB_TRY((launch_hess_y<T, 1>(dpairs.as<HessPair>(), np, x1p, x2p, dx2p,
                                             d_perm1.as<int>(), d_lab1.as<int>(),
                                             d_perm2.as<int>(), d_lab2.as<int>(), ma1, ma2, rep,
                                             W.as<T>(), Tt.as<T>(), y_scale, yth.as<__half>(),
                                             ytl.as<__half>(), nullptr, s)));
        } else {
            KFB_TRY((launch_hess_y<T, 2>(dpairs.as<HessPair>(), np, x1p, x2p, dx2p,
                                         d_perm1.as<int>(), d_lab1.as<int>(), d_perm2.as<int>(),
                                         d_lab2.as<int>(), ma1, ma2, rep, W.as<T>(), Tt.as<T>(),
                                         1.f, nullptr, nullptr, Y.as<T>(), s)));
        }
        tr_y.reset();
        auto tr_g = std::make_unique<TraceScope>("hessian:split+gemm", s);
        if (tc) {
            std::vector<TcProb> tprobs;
            tprobs.reserve(np);
            const bool narrow = ld1 <= 64;
            for (int k = 0; k < np;) {
                const HessPair &pr = pairs[p0 + k];
                const bool dg = symmetric && pr.a == pr.b;
                // merge the following pairs (a, b + 1), ... while the previous
                // molecule is whole (no padding rows between the Y blocks) and
                // the columns fit one 128-wide tile
                int k1 = k + 1, ncols = 3 * pr.nb;
                while (!dg && k1 < np) {
                    const HessPair &q = pairs[p0 + k1], &prev = pairs[p0 + k1 - 1];
                    if (q.a != pr.a || q.b != prev.b + 1 || prev.nb != ma2 ||
                        (symmetric && q.a == q.b) || ncols + 3 * q.nb > 128)
                        break;
                    ncols += 3 * q.nb;
                    ++k1;
                }
                // molecules a of at most 21 atoms: Y rows as M (up to 128 of the
                // merged pairs) and a's 3 n_a Jacobian rows as N in 64-column
                // tiles, stored transposed; else a's rows as M, Y rows as N
                TcProb p{};
                p.a_row0 = narrow ? k * ld2 : pr.a * ld1;
                p.a_k0 = 0;
                p.b_row0 = narrow ? pr.a * ld1 : k * ld2;
                p.b_k0 = 0;
                p.M = narrow ? ncols : 3 * pr.na;
                p.N = narrow ? 3 * pr.na : ncols;
                p.K = pr.na * rep;
                p.row_off = narrow ? off2[pr.b] : off1[pr.a];
                p.col_off = narrow ? off1[pr.a] : off2[pr.b];
                p.diag = dg ? 1 : 0;
                p.alpha = 1.0 / ((double)jt_scale * (double)y_scale);
                tprobs.push_back(p);
                k = k1;
            }
            TcOperand J, Yo;
            J.hi = jth.ptr;
            J.lo = jtl.ptr;
            J.rows = (long long)s1.v.nm * ld1;
            J.cols = (long long)ma1 * rep;
            Yo.hi = yth.ptr;
            Yo.lo = ytl.ptr;
            Yo.rows = (long long)np * ld2;
            Yo.cols = (long long)ma1 * rep;
            TcEpi ec;
            ec.tile_n64 = narrow ? 1 : 0;
            ec.sink_t = narrow ? 1 : 0;
            KFB_TRY(tc_gemm_grouped(narrow ? Yo : J, narrow ? J : Yo, 3, false, tprobs, sink, s,
                                    ec));
            tr_g.reset();
            if constexpr (std::is_same<T, float>::value) {
                if (hrank) {
                    TraceScope tr_r("hessian:rank", s);
                    // set-2 atoms of the batch's molecules b against the set-1
                    // Jacobian rows of its molecules a (pairs sorted by a),
                    // same label only
                    const int amin = pairs[p0].a, amax = pairs[p0 + np - 1].a;
                    std::vector<TcProb> pqs;
                    std::vector<int> qrow, qcol;
                    const long long ldq = label_problems(
                        lm2, bmin, bmax, ma2, lm1, amin, amax, ma1, ld1, rep,
                        1.0 / ((double)xs2_scale * (double)jr1_scale), pqs, qrow, qcol);
                    KFB_CUDA_TRY(cudaMemcpyAsync(d_qrow.ptr, qrow.data(),
                                                 qrow.size() * sizeof(int),
                                                 cudaMemcpyHostToDevice, s));
                    KFB_CUDA_TRY(cudaMemcpyAsync(d_qcol.ptr, qcol.data(),
                                                 qcol.size() * sizeof(int),
                                                 cudaMemcpyHostToDevice, s));
                    TcOperand Aq, Bq;
                    Aq.hi = symmetric ? x1Lh.ptr : x2Lh.ptr;
                    Aq.lo = symmetric ? x1Ll.ptr : x2Ll.ptr;
                    Aq.rows = lm2.n;
                    Aq.cols = rep;
                    Bq.hi = symmetric ? jrh.ptr : jr1h.ptr;
                    Bq.lo = symmetric ? jrl.ptr : jr1l.ptr;
                    Bq.rows = (long long)lm1.n * ld1;
                    Bq.cols = rep;
                    TcEpi eq;
                    eq.mode = EPI_DENSE;
                    eq.zf32 = d_Q.as<float>();
                    eq.ld = ldq;
                    KFB_TRY(tc_gemm_grouped(Aq, Bq, 3, false, pqs, ElemSink(), s, eq));
                    const unsigned tiles =
                        (unsigned)(((ld1 + HR_T - 1) / HR_T) * ((ld2 + HR_T - 1) / HR_T));
                    hess_rank_kernel<<<dim3(tiles, (unsigned)np), 256, 0, s>>>(
                        dpairs.as<HessPair>(), d_perm1.as<int>(), d_lab1.as<int>(),
                        d_perm2.as<int>(), d_lab2.as<int>(), ma1, ma2, d_Q.as<float>(), ldq,
                        d_qrow.as<int>(), d_qcol.as<int>(), amin, bmin,
                        symmetric ? d_pb.as<float>() : d_pb1.as<float>(), Tt.as<float>(),
                        d_off1.as<int>(), d_off2.as<int>(), symmetric ? 1 : 0, sink);
                    KFB_CUDA_TRY(cudaGetLastError());
                }
            }
            continue;
        }
        std::vector<GemmProb> probs;
        probs.reserve(np);
        for (int k = 0; k < np; ++k) {
            const HessPair &pr = pairs[p0 + k];
            GemmProb p{};
            p.A = static_cast<const T *>(s1.dx) + (size_t)pr.a * ma1 * rep * ld1;
            p.lda = ld1;
            p.transA = 1;
            p.B = Y.as<T>() + (size_t)k * ma1 * rep * ld2;
            p.ldb = ld2;
            p.M = 3 * pr.na;
            p.N = 3 * pr.nb;
            p.K = pr.na * rep;
            p.row_off = off1[pr.a];
            p.col_off = off2[pr.b];
            p.alpha = 1.0;
            p.diag = (symmetric && pr.a == pr.b) ? 1 : 0;
            probs.push_back(p);
        }
        KFB_TRY(launch_gemm<T>(probs, sink, s));
    }
    return KFB_OK;
}

template kfb_status jacobian_core<double>(const DerivSet &, const DerivSet &, int, double,
                                          double, bool, ElemSink, cudaStream_t);
template kfb_status jacobian_core<float>(const DerivSet &, const DerivSet &, int, double, double,
                                         bool, ElemSink, cudaStream_t);
template kfb_status hessian_core<double>(const DerivSet &, const DerivSet &, int, double, bool,
                                         bool, ElemSink, cudaStream_t);
template kfb_status hessian_core<float>(const DerivSet &, const DerivSet &, int, double, bool,
                                        bool, ElemSink, cudaStream_t);

}  // namespace kfb
