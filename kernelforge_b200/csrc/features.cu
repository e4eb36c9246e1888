// Element-stratified feature maps summed per molecule, on the tensor cores.
//
// * Random Fourier features (the reference's elemental RFF,
//   src/rff_elemental.hpp:7-24, GPU version src/cuda_rff_features.cu):
//     z_mol = sum over atoms a of element e: sqrt(2/D) cos(x_a . W_e + b_e)
//   x_a . W_e runs as a split-fp16 tcgen05 GEMM (hi*hi + hi*lo + lo*hi, FP32
//   accumulation); the epilogue adds b_e, takes the cosine and sums the rows
//   of each molecule before one atomic add per (molecule run, feature).
// * The learned cos-MLP map (no reference counterpart), per element e:
//     phi_e(x) = sqrt(2/D) cos(W2_e h + b2_e),   h = cos(W1_e x + b1_e)
//   with BF16 weights and activations and FP32 accumulation; layer 1's
//   epilogue writes h, layer 2's sums phi per molecule like the RFF path.
// * Its training step on same-element atom pairs,
//     loss = mean_p (phi(x_i) . phi(x_j) - exp(-|x_i - x_j|^2 / (2 sigma^2)))^2,
//   forward GEMMs with activation epilogues, the pair loss kernel, the three
//   backward GEMMs (dW2 = dZ2^T H, dH = dZ2 W2 fused with the cos derivative,
//   dW1 = dZ1^T X) and an Adam update that refreshes the BF16 weight copies.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <exception>
#include <mutex>
#include <vector>

#include "kfb_internal.h"
#include "tc_gemm.h"

using bf16 = __nv_bfloat16;

struct kfb_cosmlp {
    int nelem = 0, rep = 0, hidden = 0, d = 0, max_pairs = 0, device = 0;
    // FP32 master parameters, element-major: w1 (nelem, H, rep), b1 (nelem, H),
    // w2 (nelem, D, H), b2 (nelem, D)
    kfb::DevBuf w1, b1, w2, b2;
    kfb::DevBuf w1b, w2b, w2tb;  // BF16 copies: w1, w2 and w2 transposed (nelem, H, D)
    kfb::DevBuf mom[4], var[4];  // Adam moments per parameter tensor
    kfb::DevBuf grad[4];         // gradients of the last step (one element)
    std::vector<int> steps;      // Adam step count per element
    // batch workspace (2 Bp rows, Bp = max_pairs rounded up to 8)
    kfb::DevBuf idx, xb, xbt, z1, hb, hbt, z2, dz2, dz2t, dz1t, loss, err;
};

namespace kfb {

namespace {

constexpr float ADAM_B1 = 0.9f, ADAM_B2 = 0.999f, ADAM_EPS = 1e-8f;

long long ru8(long long v) { return (v + 7) / 8 * 8; }
unsigned nblk(long long n, int b) { return (unsigned)std::max<long long>(1, (n + b - 1) / b); }

// out[r][c] = bf16(x[idx[r]][c]) (zero row for idx < 0; idx >= nsrc gives a
// zero row and raises *bad); optionally also the transpose out_t[c * ld_t + r],
// through a 32 x 32 shared-memory tile.
template <class T>
__global__ void gather_rows_bf16_kernel(const T *__restrict__ x, long long nsrc,
                                        const int *__restrict__ idx, int nrows, int rep,
                                        bf16 *__restrict__ out, bf16 *__restrict__ out_t,
                                        long long ld_t, int *bad) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
        const int r = r0 + rr, c = c0 + threadIdx.x;
        float v = 0.f;
        if (r < nrows && c < rep) {
            const int a = idx[r];
            if (a >= nsrc) {
                if (bad) atomicExch(bad, 1);  // index outside x: zero row, reported
            } else if (a >= 0) {
                v = (float)x[(size_t)a * rep + c];
            }
            out[(size_t)r * rep + c] = __float2bfloat16_rn(v);
        }
        tile[rr][threadIdx.x] = v;
    }
    if (!out_t) return;
    __syncthreads();
    for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
        const int c = c0 + cc, r = r0 + threadIdx.x;
        if (c < rep && r < nrows)
            out_t[(size_t)c * ld_t + r] = __float2bfloat16_rn(tile[threadIdx.x][cc]);
    }
}

template <class T>
__global__ void gather_rows_f32_kernel(const T *__restrict__ x, const int *__restrict__ idx,
                                       int nrows, int rep, float *__restrict__ out) {
    const long long n = (long long)nrows * rep;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / rep), c = (int)(i % rep);
        const int a = idx[r];
        out[i] = a >= 0 ? (float)x[(size_t)a * rep + c] : 0.f;
    }
}

// dst[c * ld_dst + r] = src[r][c] for a BF16 (rows, cols) array, and
// colsum[c] += sum_r src[r][c] (FP32, optional).  64 x 64 tiles through shared
// memory; bf16x2 loads along c and bf16x2 stores along r when cols, ld_dst and
// the pointers allow it (128-byte accesses per warp), element-wise otherwise.
__global__ void transpose_bf16_kernel(const bf16 *__restrict__ src, int rows, int cols,
                                      bf16 *__restrict__ dst, long long ld_dst,
                                      float *__restrict__ colsum, int pairs) {
    __shared__ float tile[64][65];
    const int r0 = blockIdx.y * 64, c0 = blockIdx.x * 64;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    for (int rr = ty; rr < 64; rr += 8) {
        const int r = r0 + rr, c = c0 + 2 * tx;
        float v0 = 0.f, v1 = 0.f;
        if (r < rows) {
            if (pairs && c + 1 < cols) {
                const __nv_bfloat162 t =
                    *reinterpret_cast<const __nv_bfloat162 *>(src + (size_t)r * cols + c);
                v0 = __low2float(t);
                v1 = __high2float(t);
            } else {
                if (c < cols) v0 = __bfloat162float(src[(size_t)r * cols + c]);
                if (c + 1 < cols) v1 = __bfloat162float(src[(size_t)r * cols + c + 1]);
            }
        }
        tile[rr][2 * tx] = v0;
        tile[rr][2 * tx + 1] = v1;
    }
    __syncthreads();
    for (int cc = ty; cc < 64; cc += 8) {
        const int c = c0 + cc, r = r0 + 2 * tx;
        const float v0 = tile[2 * tx][cc], v1 = tile[2 * tx + 1][cc];
        if (c < cols) {
            bf16 *d = dst + (size_t)c * ld_dst + r;
            if (pairs && r + 1 < rows) {
                *reinterpret_cast<__nv_bfloat162 *>(d) = __floats2bfloat162_rn(v0, v1);
            } else {
                if (r < rows) d[0] = __float2bfloat16_rn(v0);
                if (r + 1 < rows) d[1] = __float2bfloat16_rn(v1);
            }
        }
        if (colsum) {
            float t = v0 + v1;
            for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if (tx == 0 && c < cols) atomicAdd(colsum + c, t);
        }
    }
}

kfb_status transpose_bf16(const bf16 *src, int rows, int cols, bf16 *dst, long long ld_dst,
                          float *colsum, cudaStream_t s) {
    const bool pairs = cols % 2 == 0 && ld_dst % 2 == 0 &&
                       (reinterpret_cast<uintptr_t>(src) & 3u) == 0 &&
                       (reinterpret_cast<uintptr_t>(dst) & 3u) == 0;
    transpose_bf16_kernel<<<dim3(nblk(cols, 64), nblk(rows, 64)), dim3(32, 8), 0, s>>>(
        src, rows, cols, dst, ld_dst, colsum, pairs ? 1 : 0);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

// out[r] = sum_c src[r][c] (BF16 rows, FP32 sums), one 256-thread block per
// row, 16-byte loads when the row allows them
__global__ void rowsum_bf16_kernel(const bf16 *__restrict__ src, int rows, int cols,
                                   float *__restrict__ out) {
    const int r = blockIdx.x;
    if (r >= rows) return;
    const bf16 *row = src + (size_t)r * cols;
    float t = 0.f;
    const bool vec = cols % 8 == 0 && (reinterpret_cast<uintptr_t>(row) & 15u) == 0;
    if (vec) {
        const uint4 *v = reinterpret_cast<const uint4 *>(row);
        for (int c = threadIdx.x; c < cols / 8; c += blockDim.x) {
            const uint4 u = v[c];
            const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const __nv_bfloat162 b2 = *reinterpret_cast<const __nv_bfloat162 *>(&w[q]);
                t += __low2float(b2) + __high2float(b2);
            }
        }
    } else {
        for (int c = threadIdx.x; c < cols; c += blockDim.x) t += __bfloat162float(row[c]);
    }
    __shared__ float red[32];
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        float s = 0.f;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        out[r] = s;
    }
}

// Exact pair-kernel values e_p = exp(-|x_i - x_j|^2 / (2 sigma^2)) (squared
// distance of the difference, FP64 accumulation), one warp per pair.
template <class T>
__global__ void pair_gaussian_kernel(const T *__restrict__ x, long long nsrc,
                                     const int *__restrict__ pi, const int *__restrict__ pj,
                                     int npairs, int rep, double c, float *__restrict__ out,
                                     int *bad) {
    const int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (p >= npairs) return;
    const int ia = pi[p], ib = pj[p];
    if (ia < 0 || ib < 0 || ia >= nsrc || ib >= nsrc) {
        if (lane == 0) {
            out[p] = 0.f;
            atomicExch(bad, 1);
        }
        return;
    }
    const T *a = x + (size_t)ia * rep;
    const T *b = x + (size_t)ib * rep;
    double t = 0.0;
    for (int k = lane; k < rep; k += 32) {
        const double d = (double)a[k] - (double)b[k];
        t += d * d;
    }
    for (int o = 16; o; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) out[p] = (float)exp(c * t);
}

// sin and cos of x: reduce to r = x - 2 pi round(x / 2 pi) in [-pi, pi] (2 pi
// split into a float head and tail so the product is exact to ~1e-7 for the
// |x| < 1e3 the network produces), then the hardware approximation, whose
// absolute error on [-pi, pi] is about 1e-6.
__device__ __forceinline__ void sincos_reduced(float x, float &sn, float &cs) {
    const float TWO_PI_HI = 6.28318548202514648f;     // float(2 pi)
    const float TWO_PI_LO = -1.74845553e-07f;          // 2 pi - TWO_PI_HI
    const float k = rintf(x * 0.159154943091895336f);  // x / (2 pi)
    const float r = fmaf(-k, TWO_PI_LO, fmaf(-k, TWO_PI_HI, x));
    __sincosf(r, &sn, &cs);
}

// Pair loss and the gradient at layer 2's pre-activation.  Rows p and p + Bp
// of z2 are the two atoms of pair p.  With s2 = 2 / D:
//   k_p = s2 sum_d cos z_i[d] cos z_j[d],  r_p = k_p - t_p,  loss += r_p^2
//   dZ2_i[d] = -(2 r_p / npairs) s2 cos z_j[d] sin z_i[d]   (and i <-> j)
// Padded pairs (p >= npairs) get zero gradient rows.  One block of 256
// threads per pair; each thread keeps its float4 slices of both rows in
// registers between the dot product and the gradient (D <= 256 * 4 * VPT).
constexpr int PL_THREADS = 256, PL_VPT = 4;
__global__ void __launch_bounds__(PL_THREADS)
    pair_loss_kernel(const float *__restrict__ z2, int Bp, int npairs, int D,
                     const float *__restrict__ target, float s2, float gscale,
                     bf16 *__restrict__ dz2, double *__restrict__ loss) {
    const int p = blockIdx.x;
    const float4 *zi = reinterpret_cast<const float4 *>(z2 + (size_t)p * D);
    const float4 *zj = reinterpret_cast<const float4 *>(z2 + (size_t)(p + Bp) * D);
    uint2 *di = reinterpret_cast<uint2 *>(dz2 + (size_t)p * D);
    uint2 *dj = reinterpret_cast<uint2 *>(dz2 + (size_t)(p + Bp) * D);
    const int n4 = D / 4;
    if (p >= npairs) {
        for (int k = threadIdx.x; k < n4; k += PL_THREADS) {
            di[k] = make_uint2(0u, 0u);
            dj[k] = make_uint2(0u, 0u);
        }
        return;
    }
    // sin / cos of both rows once, kept in registers between the dot product
    // and the gradient
    float si[PL_VPT][4], ci[PL_VPT][4], sj[PL_VPT][4], cj[PL_VPT][4];
    float acc = 0.f;
#pragma unroll
    for (int u = 0; u < PL_VPT; ++u) {
        const int k = threadIdx.x + u * PL_THREADS;
        if (k < n4) {
            const float4 a = zi[k], b = zj[k];
            const float av[4] = {a.x, a.y, a.z, a.w}, bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                sincos_reduced(av[c], si[u][c], ci[u][c]);
                sincos_reduced(bv[c], sj[u][c], cj[u][c]);
                acc = fmaf(ci[u][c], cj[u][c], acc);
            }
        }
    }
    __shared__ float red[PL_THREADS / 32];
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    float tot = 0.f;
#pragma unroll
    for (int w = 0; w < PL_THREADS / 32; ++w) tot += red[w];
    const float r = s2 * tot - target[p];
    if (threadIdx.x == 0) atomicAdd(loss, (double)r * (double)r);
    const float g = gscale * r * s2;
#pragma unroll
    for (int u = 0; u < PL_VPT; ++u) {
        const int k = threadIdx.x + u * PL_THREADS;
        if (k < n4) {
            const __nv_bfloat162 x01 = __floats2bfloat162_rn(-g * cj[u][0] * si[u][0],
                                                             -g * cj[u][1] * si[u][1]);
            const __nv_bfloat162 x23 = __floats2bfloat162_rn(-g * cj[u][2] * si[u][2],
                                                             -g * cj[u][3] * si[u][3]);
            const __nv_bfloat162 y01 = __floats2bfloat162_rn(-g * ci[u][0] * sj[u][0],
                                                             -g * ci[u][1] * sj[u][1]);
            const __nv_bfloat162 y23 = __floats2bfloat162_rn(-g * ci[u][2] * sj[u][2],
                                                             -g * ci[u][3] * sj[u][3]);
            di[k] = make_uint2(*reinterpret_cast<const uint32_t *>(&x01),
                               *reinterpret_cast<const uint32_t *>(&x23));
            dj[k] = make_uint2(*reinterpret_cast<const uint32_t *>(&y01),
                               *reinterpret_cast<const uint32_t *>(&y23));
        }
    }
}

// Adam on one parameter tensor (n values), refreshing its BF16 copy (pb)
// when given.
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, long long n, float lr,
                            float bc1, float bc2, bf16 *__restrict__ pb) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = ADAM_B1 * m[i] + (1.f - ADAM_B1) * gi;
        const float vi = ADAM_B2 * v[i] + (1.f - ADAM_B2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + ADAM_EPS);
        p[i] = pi;
        if (pb) pb[i] = __float2bfloat16_rn(pi);
    }
}

__global__ void to_bf16_kernel(const float *__restrict__ p, int rows, int cols,
                               bf16 *__restrict__ pb, bf16 *__restrict__ pbt) {
    const long long n = (long long)rows * cols;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const bf16 h = __float2bfloat16_rn(p[i]);
        if (pb) pb[i] = h;
        if (pbt) pbt[(i % cols) * rows + i / cols] = h;
    }
}

// Atoms of each element in molecule order: flat padded indices m * ma + j and
// the molecule of each row.
struct ElemRows {
    std::vector<std::vector<int>> idx, mol;
};

kfb_status elem_rows(const int *q, const int *n, int nm, int ma, int nelem, ElemRows &er) {
    er.idx.assign(nelem, {});
    er.mol.assign(nelem, {});
    for (int m = 0; m < nm; ++m) {
        const int na = std::min(std::max(n[m], 0), ma);
        for (int j = 0; j < na; ++j) {
            const int e = q[(size_t)m * ma + j];
            if (e < 0) continue;
            if (e >= nelem)
                return set_error(KFB_ERR_INVALID_ARG,
                                 "element index %d out of range [0, %d) (molecule %d, atom %d)", e,
                                 nelem, m, j);
            er.idx[e].push_back(m * ma + j);
            er.mol[e].push_back(m);
        }
    }
    return KFB_OK;
}

size_t feature_budget() {
    static size_t b = [] {
        const char *v = std::getenv("KFB_WORKSPACE_GB");
        double gb = v ? std::atof(v) : 4.0;
        if (!(gb > 0)) gb = 4.0;
        return (size_t)(gb * (1ull << 30));
    }();
    return b;
}

// ---------------------------------------------------------------- RFF forces
// K-padded operands for the force path (the tensor-core GEMM needs K % 16 == 0):
// dst (rows, kpad) with dst[r][k] = src row r (stride src_ld) for k < rep, else 0.
template <class T>
__global__ void gather_pad_rows_kernel(const T *__restrict__ x, const int *__restrict__ idx,
                                       int nrows, int rep, int kpad, float *__restrict__ out) {
    const long long n = (long long)nrows * kpad;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(i / kpad), k = (int)(i % kpad);
        out[i] = k < rep ? (float)x[(size_t)idx[r] * rep + k] : 0.f;
    }
}

// wt (d, kpad) = W_e^T, zero beyond rep
__global__ void transpose_pad_kernel(const float *__restrict__ w, int rep, int d, int kpad,
                                     float *__restrict__ wt) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int rr = r0 + r, cc = c0 + threadIdx.x;
        tile[r][threadIdx.x] = (rr < rep && cc < d) ? w[(size_t)rr * d + cc] : 0.f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int cc = c0 + r, rr = r0 + threadIdx.x;  // output row cc (feature), column rr
        if (cc < d && rr < kpad) wt[(size_t)cc * kpad + rr] = tile[threadIdx.x][r];
    }
}

// Jacobian rows: out[r][k] = dx[(src[r] * rep + k) * ld + col[r]] (k < rep), 0 beyond
template <class T>
__global__ void jacobian_rows_kernel(const T *__restrict__ dx, const int *__restrict__ src,
                                     const int *__restrict__ col, int nrows, int rep, int ld,
                                     int kpad, float *__restrict__ out) {
    const int r = blockIdx.x;
    if (r >= nrows) return;
    const T *base = dx + (size_t)src[r] * rep * ld + col[r];
    for (int k = threadIdx.x; k < kpad; k += blockDim.x)
        out[(size_t)r * kpad + k] = k < rep ? (float)base[(size_t)k * ld] : 0.f;
}

template <class T>
kfb_status rff_features_t(const T *x, const int *q, const int *n, int nm, int ma, int rep,
                          const float *w, const float *b, int nelem, int d, float *z,
                          cudaStream_t s) {
    KFB_TRY(zero(z, (size_t)nm * d * sizeof(float), s));
    ElemRows er;
    KFB_TRY(elem_rows(q, n, nm, ma, nelem, er));
    // W_e^T (d, kpad) split once per element; K padded with zeros to a multiple of 16
    const int kpad = (rep + 15) / 16 * 16;
    DevBuf wt, wh, wl;
    KFB_TRY(wt.alloc((size_t)d * kpad * sizeof(float), s));
    KFB_TRY(wh.alloc((size_t)d * kpad * sizeof(__half), s));
    KFB_TRY(wl.alloc((size_t)d * kpad * sizeof(__half), s));
    const size_t row_bytes = (size_t)kpad * (sizeof(float) + 2 * sizeof(__half));
    const int chunk = (int)std::max<size_t>(128, feature_budget() / row_bytes);
    DevBuf xr, xh, xl, didx, dmol;
    const float sc = std::sqrt(2.f / (float)d);
    for (int e = 0; e < nelem; ++e) {
        const int ne = (int)er.idx[e].size();
        if (ne == 0) continue;
        transpose_pad_kernel<<<dim3(nblk(d, 32), nblk(kpad, 32)), dim3(32, 8), 0, s>>>(
            w + (size_t)e * rep * d, rep, d, kpad, wt.as<float>());
        KFB_CUDA_TRY(cudaGetLastError());
        float w_scale = 1.f;
        KFB_TRY(split_rows<float>(wt.as<float>(), (long long)d * kpad, wh.as<__half>(),
                                  wl.as<__half>(), &w_scale, s));
        KFB_TRY(upload(didx, er.idx[e], s));
        KFB_TRY(upload(dmol, er.mol[e], s));
        const int rows_max = std::min(ne, chunk);
        KFB_TRY(xr.alloc((size_t)rows_max * kpad * sizeof(float), s));
        KFB_TRY(xh.alloc((size_t)rows_max * kpad * sizeof(__half), s));
        KFB_TRY(xl.alloc((size_t)rows_max * kpad * sizeof(__half), s));
        for (int r0 = 0; r0 < ne; r0 += chunk) {
            const int nr = std::min(chunk, ne - r0);
            gather_pad_rows_kernel<T><<<nblk((long long)nr * kpad, 256 * 8), 256, 0, s>>>(
                x, didx.as<int>() + r0, nr, rep, kpad, xr.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            float x_scale = 1.f;
            KFB_TRY(split_rows<float>(xr.as<float>(), (long long)nr * kpad, xh.as<__half>(),
                                      xl.as<__half>(), &x_scale, s));
            TcOperand A, B;
            A.hi = xh.ptr;
            A.lo = xl.ptr;
            A.rows = nr;
            A.cols = kpad;
            B.hi = wh.ptr;
            B.lo = wl.ptr;
            B.rows = d;
            B.cols = kpad;
            TcProb p{};
            p.M = nr;
            p.N = d;
            p.K = kpad;
            p.row_off = 0;
            p.alpha = 1.0 / ((double)x_scale * (double)w_scale);
            TcEpi epi;
            epi.mode = EPI_COS_MOLSUM;
            epi.bias = b + (size_t)e * d;
            epi.mol = dmol.as<int>() + r0;
            epi.molsum = z;
            epi.ld = d;
            epi.scale = sc;
            KFB_TRY(tc_gemm_grouped(A, B, 3, false, {p}, ElemSink(), s, epi));
        }
    }
    return KFB_OK;
}

// G (naq, d) += rows 3 off_m + c: sqrt(2/d) sum_j sin(z_j) (W_e^T dX[m, j, :, c]), z_j the
// pre-activation x_j W_e + b_e (src/rff_elemental.cpp:363-500 stores the transpose).
template <class T>
kfb_status rff_gradient_t(const T *x, const T *dx, const int *q, const int *n, int nm, int ma,
                          int rep, const float *w, const float *b, int nelem, int d, float *g,
                          cudaStream_t s) {
    std::vector<int> offs(nm + 1, 0);
    for (int m = 0; m < nm; ++m) offs[m + 1] = offs[m] + 3 * std::min(std::max(n[m], 0), ma);
    KFB_TRY(zero(g, (size_t)std::max(offs[nm], 1) * d * sizeof(float), s));
    ElemRows er;
    KFB_TRY(elem_rows(q, n, nm, ma, nelem, er));
    const int kpad = (rep + 15) / 16 * 16, ld = 3 * ma;
    DevBuf wt, wh, wl;
    KFB_TRY(wt.alloc((size_t)d * kpad * sizeof(float), s));
    KFB_TRY(wh.alloc((size_t)d * kpad * sizeof(__half), s));
    KFB_TRY(wl.alloc((size_t)d * kpad * sizeof(__half), s));
    // per atom: one Z row (d floats) and up to 3 ma Jacobian rows (kpad wide, FP32 + pair)
    const size_t atom_bytes = (size_t)d * sizeof(float) +
                              (size_t)(1 + ld) * kpad * (sizeof(float) + 2 * sizeof(__half));
    const int chunk = (int)std::max<size_t>(1, feature_budget() / atom_bytes);
    const float sc = std::sqrt(2.f / (float)d);
    DevBuf zpre, xr, xh, xl, jr, jh, jl, didx, dsrc, dcol, ddst, daux;
    for (int e = 0; e < nelem; ++e) {
        const int ne = (int)er.idx[e].size();
        if (ne == 0) continue;
        transpose_pad_kernel<<<dim3(nblk(d, 32), nblk(kpad, 32)), dim3(32, 8), 0, s>>>(
            w + (size_t)e * rep * d, rep, d, kpad, wt.as<float>());
        KFB_CUDA_TRY(cudaGetLastError());
        float w_scale = 1.f;
        KFB_TRY(split_rows<float>(wt.as<float>(), (long long)d * kpad, wh.as<__half>(),
                                  wl.as<__half>(), &w_scale, s));
        TcOperand B;
        B.hi = wh.ptr;
        B.lo = wl.ptr;
        B.rows = d;
        B.cols = kpad;
        for (int a0 = 0; a0 < ne; a0 += chunk) {
            const int na = std::min(chunk, ne - a0);
            // rows of the chunk, ordered (molecule, c, atom): one destination per run
            std::vector<int> src, col, dst, aux;
            for (int t = 0; t < na;) {
                const int m = er.mol[e][a0 + t];
                int t1 = t;
                while (t1 < na && er.mol[e][a0 + t1] == m) ++t1;
                const int nc = offs[m + 1] - offs[m];
                for (int c = 0; c < nc; ++c)
                    for (int u = t; u < t1; ++u) {
                        src.push_back(er.idx[e][a0 + u]);
                        col.push_back(c);
                        dst.push_back(offs[m] + c);
                        aux.push_back(u);
                    }
                t = t1;
            }
            const int nr = (int)src.size();
            std::vector<int> aidx(er.idx[e].begin() + a0, er.idx[e].begin() + a0 + na);
            KFB_TRY(upload(didx, aidx, s));
            KFB_TRY(upload(dsrc, src, s));
            KFB_TRY(upload(dcol, col, s));
            KFB_TRY(upload(ddst, dst, s));
            KFB_TRY(upload(daux, aux, s));
            // pre-activations Z = X_e W_e + b_e (na, d), FP32
            KFB_TRY(zpre.alloc((size_t)na * d * sizeof(float), s));
            KFB_TRY(xr.alloc((size_t)na * kpad * sizeof(float), s));
            KFB_TRY(xh.alloc((size_t)na * kpad * sizeof(__half), s));
            KFB_TRY(xl.alloc((size_t)na * kpad * sizeof(__half), s));
            gather_pad_rows_kernel<T><<<nblk((long long)na * kpad, 256 * 8), 256, 0, s>>>(
                x, didx.as<int>(), na, rep, kpad, xr.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            float x_scale = 1.f;
            KFB_TRY(split_rows<float>(xr.as<float>(), (long long)na * kpad, xh.as<__half>(),
                                      xl.as<__half>(), &x_scale, s));
            {
                TcOperand A;
                A.hi = xh.ptr;
                A.lo = xl.ptr;
                A.rows = na;
                A.cols = kpad;
                TcProb p{};
                p.M = na;
                p.N = d;
                p.K = kpad;
                p.alpha = 1.0 / ((double)x_scale * (double)w_scale);
                TcEpi epi;
                epi.mode = EPI_DENSE;
                epi.zf32 = zpre.as<float>();
                epi.bias = b + (size_t)e * d;
                epi.ld = d;
                KFB_TRY(tc_gemm_grouped(A, B, 3, false, {p}, ElemSink(), s, epi));
            }
            // Jacobian rows (nr, kpad) times W_e, weighted by sqrt(2/d) sin(Z) and
            // summed into G per destination row
            KFB_TRY(jr.alloc((size_t)nr * kpad * sizeof(float), s));
            KFB_TRY(jh.alloc((size_t)nr * kpad * sizeof(__half), s));
            KFB_TRY(jl.alloc((size_t)nr * kpad * sizeof(__half), s));
            jacobian_rows_kernel<T><<<nr, 128, 0, s>>>(dx, dsrc.as<int>(), dcol.as<int>(), nr, rep,
                                                       ld, kpad, jr.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
            float j_scale = 1.f;
            KFB_TRY(split_rows<float>(jr.as<float>(), (long long)nr * kpad, jh.as<__half>(),
                                      jl.as<__half>(), &j_scale, s));
            TcOperand A;
            A.hi = jh.ptr;
            A.lo = jl.ptr;
            A.rows = nr;
            A.cols = kpad;
            TcProb p{};
            p.M = nr;
            p.N = d;
            p.K = kpad;
            p.alpha = 1.0 / ((double)j_scale * (double)w_scale);
            TcEpi epi;
            epi.mode = EPI_SIN_RUNSUM;
            epi.mol = ddst.as<int>();
            epi.atom = daux.as<int>();
            epi.aux = zpre.as<float>();
            epi.ld_aux = d;
            epi.molsum = g;
            epi.ld = d;
            epi.scale = sc;
            KFB_TRY(tc_gemm_grouped(A, B, 3, false, {p}, ElemSink(), s, epi));
        }
    }
    return KFB_OK;
}

kfb_status check_cosmlp(const kfb_cosmlp *h) {
    if (!h) return set_error(KFB_ERR_INVALID_ARG, "null cos-MLP handle");
    int dev = 0;
    KFB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev != h->device)
        return set_error(KFB_ERR_INVALID_ARG, "cos-MLP handle belongs to device %d, current is %d",
                         h->device, dev);
    return KFB_OK;
}

template <class T>
kfb_status cosmlp_features_t(kfb_cosmlp *h, const T *x, const int *q, const int *n, int nm,
                             int ma, float *z, cudaStream_t s) {
    const int rep = h->rep, H = h->hidden, D = h->d;
    KFB_TRY(zero(z, (size_t)nm * D * sizeof(float), s));
    ElemRows er;
    KFB_TRY(elem_rows(q, n, nm, ma, h->nelem, er));
    const size_t row_bytes = (size_t)(rep + H) * sizeof(bf16);
    const int chunk = (int)std::max<size_t>(128, feature_budget() / row_bytes);
    DevBuf xb, hb, didx, dmol;
    const float sc = std::sqrt(2.f / (float)D);
    for (int e = 0; e < h->nelem; ++e) {
        const int ne = (int)er.idx[e].size();
        if (ne == 0) continue;
        KFB_TRY(upload(didx, er.idx[e], s));
        KFB_TRY(upload(dmol, er.mol[e], s));
        const int rows_max = std::min(ne, chunk);
        KFB_TRY(xb.alloc((size_t)rows_max * rep * sizeof(bf16), s));
        KFB_TRY(hb.alloc((size_t)rows_max * H * sizeof(bf16), s));
        for (int r0 = 0; r0 < ne; r0 += chunk) {
            const int nr = std::min(chunk, ne - r0);
            gather_rows_bf16_kernel<T><<<dim3(nblk(rep, 32), nblk(nr, 32)), dim3(32, 8), 0, s>>>(
                x, (long long)nm * ma, didx.as<int>() + r0, nr, rep, xb.as<bf16>(), nullptr, 0,
                nullptr);
            KFB_CUDA_TRY(cudaGetLastError());
            TcOperand A, B;
            A.hi = xb.ptr;
            A.rows = nr;
            A.cols = rep;
            B.hi = h->w1b.ptr;
            B.rows = (long long)h->nelem * H;
            B.cols = rep;
            TcProb p{};
            p.b_row0 = e * H;
            p.M = nr;
            p.N = H;
            p.K = rep;
            p.alpha = 1.0;
            TcEpi e1;
            e1.mode = EPI_DENSE;
            e1.bias = h->b1.as<float>() + (size_t)e * H;
            e1.act = hb.as<bf16>();
            e1.ld = H;
            KFB_TRY(tc_gemm_grouped(A, B, 1, true, {p}, ElemSink(), s, e1));
            TcOperand A2, B2;
            A2.hi = hb.ptr;
            A2.rows = nr;
            A2.cols = H;
            B2.hi = h->w2b.ptr;
            B2.rows = (long long)h->nelem * D;
            B2.cols = H;
            TcProb p2{};
            p2.b_row0 = e * D;
            p2.M = nr;
            p2.N = D;
            p2.K = H;
            p2.alpha = 1.0;
            TcEpi e2;
            e2.mode = EPI_COS_MOLSUM;
            e2.bias = h->b2.as<float>() + (size_t)e * D;
            e2.mol = dmol.as<int>() + r0;
            e2.molsum = z;
            e2.ld = D;
            e2.scale = sc;
            KFB_TRY(tc_gemm_grouped(A2, B2, 1, true, {p2}, ElemSink(), s, e2));
        }
    }
    return KFB_OK;
}

template <class T>
kfb_status cosmlp_step_t(kfb_cosmlp *h, int e, const T *x, long long nrows, const int *pi,
                         const int *pj, const float *target, int npairs, float lr, int update,
                         double *loss_out, cudaStream_t s) {
    const int rep = h->rep, H = h->hidden, D = h->d;
    const int Bp = (int)ru8(npairs);
    const int R = 2 * Bp;  // batch rows: i-atoms then j-atoms
    int *err = h->err.as<int>();
    KFB_TRY(zero(err, sizeof(int), s));
    KFB_TRY(zero(h->loss.ptr, sizeof(double), s));
    // batch row indices: pi, padding, pj, padding
    int *idx = h->idx.as<int>();
    KFB_CUDA_TRY(cudaMemsetAsync(idx, 0xff, (size_t)R * sizeof(int), s));
    KFB_CUDA_TRY(cudaMemcpyAsync(idx, pi, (size_t)npairs * sizeof(int), cudaMemcpyDeviceToDevice, s));
    KFB_CUDA_TRY(cudaMemcpyAsync(idx + Bp, pj, (size_t)npairs * sizeof(int),
                                 cudaMemcpyDeviceToDevice, s));
    int *bad = h->err.as<int>() + 1;
    KFB_TRY(zero(bad, sizeof(int), s));
    gather_rows_bf16_kernel<T><<<dim3(nblk(rep, 32), nblk(R, 32)), dim3(32, 8), 0, s>>>(
        x, nrows, idx, R, rep, h->xb.as<bf16>(), h->xbt.as<bf16>(), R, bad);
    KFB_CUDA_TRY(cudaGetLastError());
    // forward, layer 1: z1 = X W1^T + b1, h = cos z1 (rows and transposed)
    {
        TcOperand A, B;
        A.hi = h->xb.ptr;
        A.rows = R;
        A.cols = rep;
        B.hi = h->w1b.ptr;
        B.rows = (long long)h->nelem * H;
        B.cols = rep;
        TcProb p{};
        p.b_row0 = e * H;
        p.M = R;
        p.N = H;
        p.K = rep;
        p.alpha = 1.0;
        TcEpi ep;
        ep.mode = EPI_DENSE;
        ep.bias = h->b1.as<float>() + (size_t)e * H;
        ep.zf32 = h->z1.as<float>();
        ep.act = h->hb.as<bf16>();
        ep.act_t = h->hbt.as<bf16>();
        ep.ld = H;
        ep.ld_t = R;
        KFB_TRY(tc_gemm_grouped(A, B, 1, true, {p}, ElemSink(), s, ep, err));
    }
    // forward, layer 2: z2 = h W2^T + b2
    {
        TcOperand A, B;
        A.hi = h->hb.ptr;
        A.rows = R;
        A.cols = H;
        B.hi = h->w2b.ptr;
        B.rows = (long long)h->nelem * D;
        B.cols = H;
        TcProb p{};
        p.b_row0 = e * D;
        p.M = R;
        p.N = D;
        p.K = H;
        p.alpha = 1.0;
        TcEpi ep;
        ep.mode = EPI_DENSE;
        ep.bias = h->b2.as<float>() + (size_t)e * D;
        ep.zf32 = h->z2.as<float>();
        ep.ld = D;
        KFB_TRY(tc_gemm_grouped(A, B, 1, true, {p}, ElemSink(), s, ep, err));
    }
    float *gw1 = h->grad[0].as<float>(), *gb1 = h->grad[1].as<float>();
    float *gw2 = h->grad[2].as<float>(), *gb2 = h->grad[3].as<float>();
    pair_loss_kernel<<<Bp, PL_THREADS, 0, s>>>(h->z2.as<float>(), Bp, npairs, D, target,
                                               2.f / (float)D, 2.f / (float)npairs,
                                               h->dz2.as<bf16>(), h->loss.as<double>());
    KFB_CUDA_TRY(cudaGetLastError());
    KFB_TRY(zero(gb2, (size_t)D * sizeof(float), s));
    KFB_TRY(transpose_bf16(h->dz2.as<bf16>(), R, D, h->dz2t.as<bf16>(), R, gb2, s));
    // dW2 = dZ2^T H  (D x H, contraction over the batch rows)
    {
        TcOperand A, B;
        A.hi = h->dz2t.ptr;
        A.rows = D;
        A.cols = R;
        B.hi = h->hbt.ptr;
        B.rows = H;
        B.cols = R;
        TcProb p{};
        p.M = D;
        p.N = H;
        p.K = R;
        p.alpha = 1.0;
        TcEpi ep;
        ep.mode = EPI_DENSE;
        ep.zf32 = gw2;
        ep.ld = H;
        KFB_TRY(tc_gemm_grouped(A, B, 1, true, {p}, ElemSink(), s, ep, err));
    }
    // dZ1 = (dZ2 W2) * -sin z1, written transposed (H x R)
    {
        TcOperand A, B;
        A.hi = h->dz2.ptr;
        A.rows = R;
        A.cols = D;
        B.hi = h->w2tb.ptr;
        B.rows = (long long)h->nelem * H;
        B.cols = D;
        TcProb p{};
        p.b_row0 = e * H;
        p.M = R;
        p.N = H;
        p.K = D;
        p.alpha = 1.0;
        TcEpi ep;
        ep.mode = EPI_DSIN_T;
        ep.aux = h->z1.as<float>();
        ep.ld = H;
        ep.act_t = h->dz1t.as<bf16>();
        ep.ld_t = R;
        KFB_TRY(tc_gemm_grouped(A, B, 1, true, {p}, ElemSink(), s, ep, err));
    }
    // dW1 = dZ1^T X  (H x rep): few output tiles, so the batch axis (K) is
    // split over problems that add into a zeroed gradient
    {
        TcOperand A, B;
        A.hi = h->dz1t.ptr;
        A.rows = H;
        A.cols = R;
        B.hi = h->xbt.ptr;
        B.rows = rep;
        B.cols = R;
        const int tiles = ((H + 127) / 128) * ((rep + 127) / 128);
        const int want = std::max(1, std::min(device_sm_count() / std::max(tiles, 1), R / 256));
        const int kc = (int)((R / want + 63) / 64 * 64);
        std::vector<TcProb> probs;
        for (int k0 = 0; k0 < R; k0 += kc) {
            TcProb p{};
            p.a_k0 = p.b_k0 = k0;
            p.M = H;
            p.N = rep;
            p.K = std::min(kc, R - k0);
            p.alpha = 1.0;
            probs.push_back(p);
        }
        TcEpi ep;
        ep.mode = EPI_DENSE;
        ep.zf32 = gw1;
        ep.ld = rep;
        ep.accumulate = probs.size() > 1 ? 1 : 0;
        if (ep.accumulate) KFB_TRY(zero(gw1, (size_t)H * rep * sizeof(float), s));
        KFB_TRY(tc_gemm_grouped(A, B, 1, true, probs, ElemSink(), s, ep, err));
    }
    rowsum_bf16_kernel<<<H, 256, 0, s>>>(h->dz1t.as<bf16>(), H, R, gb1);
    KFB_CUDA_TRY(cudaGetLastError());
    if (update) {
        const int t = ++h->steps[e];
        const float bc1 = 1.f - std::pow(ADAM_B1, (float)t);
        const float bc2 = 1.f - std::pow(ADAM_B2, (float)t);
        struct P {
            DevBuf *p;
            int k, rows, cols;
            bf16 *pb, *pbt;
        };
        const P ps[4] = {
            {&h->w1, 0, H, rep, h->w1b.as<bf16>() + (size_t)e * H * rep, nullptr},
            {&h->b1, 1, 1, H, nullptr, nullptr},
            {&h->w2, 2, D, H, h->w2b.as<bf16>() + (size_t)e * D * H,
             h->w2tb.as<bf16>() + (size_t)e * H * D},
            {&h->b2, 3, 1, D, nullptr, nullptr},
        };
        for (const P &q : ps) {
            const size_t off = (size_t)e * q.rows * q.cols;
            const long long n = (long long)q.rows * q.cols;
            adam_kernel<<<nblk(n, 256 * 4), 256, 0, s>>>(
                q.p->as<float>() + off, h->grad[q.k].as<float>(), h->mom[q.k].as<float>() + off,
                h->var[q.k].as<float>() + off, n, lr, bc1, bc2, q.pb);
            KFB_CUDA_TRY(cudaGetLastError());
            if (q.pbt) KFB_TRY(transpose_bf16(q.pb, q.rows, q.cols, q.pbt, q.rows, nullptr, s));
        }
    }
    int herr[2] = {0, 0};
    double lsum = 0.0;
    KFB_CUDA_TRY(cudaMemcpyAsync(herr, err, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaMemcpyAsync(&lsum, h->loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr[0]) return set_error(KFB_ERR_TIMEOUT, "cos-MLP step: a tensor-core pipeline wait timed out");
    if (herr[1])
        return set_error(KFB_ERR_INVALID_ARG,
                         "cos-MLP step: a pair index is outside the %lld rows of x (the step "
                         "used zero rows for it; parameters were %s)",
                         nrows, update ? "updated" : "not updated");
    if (loss_out) *loss_out = lsum / std::max(npairs, 1);
    return KFB_OK;
}

}  // namespace

}  // namespace kfb

using namespace kfb;

namespace {
// Host allocations (std::vector) may throw; no exception crosses the C ABI.
template <class F>
kfb_status guarded(F &&f) {
    try {
        return f();
    } catch (const std::exception &ex) {
        return set_error(KFB_ERR_ALLOC, "host exception: %s", ex.what());
    }
}
}  // namespace

extern "C" {

kfb_status kfb_rff_features_elemental(const void *x, const int *q, const int *n, int nm, int ma,
                                      int rep, const float *w, const float *b, int nelem, int d,
                                      kfb_dtype x_dtype, float *z, void *stream) {
    return guarded([&]() -> kfb_status {
        if (!x || !q || !n || !w || !b || !z)
            return set_error(KFB_ERR_INVALID_ARG, "null pointer argument");
        if (nm <= 0 || ma <= 0 || rep <= 0 || nelem <= 0 || d <= 0)
            return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
        if (d % 8 != 0)
            return set_error(KFB_ERR_UNSUPPORTED,
                             "rff_features_elemental: D must be a multiple of 8");
        if (!device_is_sm100())
            return set_error(KFB_ERR_UNSUPPORTED, "feature maps need an sm_100 (B200) device");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (x_dtype == KFB_F64)
            return rff_features_t<double>(static_cast<const double *>(x), q, n, nm, ma, rep, w,
                                          b, nelem, d, z, s);
        return rff_features_t<float>(static_cast<const float *>(x), q, n, nm, ma, rep, w, b,
                                     nelem, d, z, s);
    });
}

kfb_status kfb_rff_gradient_elemental(const void *x, const void *dx, const int *q, const int *n,
                                      int nm, int ma, int rep, const float *w, const float *b,
                                      int nelem, int d, kfb_dtype x_dt, float *g, void *stream) {
    return guarded([&]() -> kfb_status {
        if (!x || !dx || !q || !n || !w || !b || !g)
            return set_error(KFB_ERR_INVALID_ARG, "null pointer");
        if (nm <= 0 || ma <= 0 || rep <= 0 || nelem <= 0 || d <= 0)
            return set_error(KFB_ERR_INVALID_ARG, "dimensions must be positive");
        if (d % 8 != 0) return set_error(KFB_ERR_INVALID_ARG, "D must be a multiple of 8");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (x_dt == KFB_F64)
            return rff_gradient_t<double>(static_cast<const double *>(x),
                                          static_cast<const double *>(dx), q, n, nm, ma, rep, w,
                                          b, nelem, d, g, s);
        return rff_gradient_t<float>(static_cast<const float *>(x), static_cast<const float *>(dx),
                                     q, n, nm, ma, rep, w, b, nelem, d, g, s);
    });
}

kfb_status kfb_pair_gaussian(const void *x, long long nrows, const int *pi, const int *pj,
                             int npairs, int rep, double sigma, kfb_dtype x_dtype, float *out,
                             void *stream) {
    if (!x || !pi || !pj || !out) return set_error(KFB_ERR_INVALID_ARG, "null pointer argument");
    if (npairs < 0 || rep <= 0 || nrows <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    if (!(sigma > 0)) return set_error(KFB_ERR_INVALID_ARG, "sigma must be > 0");
    if (npairs == 0) return KFB_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DevBuf bad;
    KFB_TRY(bad.alloc(sizeof(int), s));
    KFB_TRY(zero(bad.ptr, sizeof(int), s));
    const double c = -1.0 / (2.0 * sigma * sigma);
    if (x_dtype == KFB_F64)
        pair_gaussian_kernel<double><<<nblk(npairs, 8), 256, 0, s>>>(
            static_cast<const double *>(x), nrows, pi, pj, npairs, rep, c, out, bad.as<int>());
    else
        pair_gaussian_kernel<float><<<nblk(npairs, 8), 256, 0, s>>>(
            static_cast<const float *>(x), nrows, pi, pj, npairs, rep, c, out, bad.as<int>());
    KFB_CUDA_TRY(cudaGetLastError());
    int hb = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&hb, bad.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (hb)
        return set_error(KFB_ERR_INVALID_ARG,
                         "pair_gaussian: a pair index is outside the %lld rows of x", nrows);
    return KFB_OK;
}

kfb_status kfb_cosmlp_create(int nelem, int rep, int hidden, int d, int max_pairs,
                             kfb_cosmlp **out) {
    return guarded([&]() -> kfb_status {
        if (!out) return set_error(KFB_ERR_INVALID_ARG, "null output handle pointer");
        *out = nullptr;
        if (nelem <= 0 || rep <= 0 || hidden <= 0 || d <= 0 || max_pairs <= 0)
            return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
        if (rep % 16 != 0 || hidden % 16 != 0 || d % 16 != 0)
            return set_error(KFB_ERR_UNSUPPORTED,
                             "cos-MLP: rep, hidden and D must be multiples of 16");
        if (d > PL_THREADS * 4 * PL_VPT)
            return set_error(KFB_ERR_UNSUPPORTED, "cos-MLP: D up to %d", PL_THREADS * 4 * PL_VPT);
        if (!device_is_sm100())
            return set_error(KFB_ERR_UNSUPPORTED, "cos-MLP needs an sm_100 (B200) device");
        auto *h = new kfb_cosmlp();
        h->nelem = nelem;
        h->rep = rep;
        h->hidden = hidden;
        h->d = d;
        h->max_pairs = max_pairs;
        h->steps.assign(nelem, 0);
        kfb_status st = KFB_OK;
        auto fail = [&](kfb_status v) {
            delete h;
            return v;
        };
        if ((st = [&]() -> kfb_status {
                 KFB_CUDA_TRY(cudaGetDevice(&h->device));
                 cudaStream_t s = nullptr;
                 const size_t n1 = (size_t)nelem * hidden * rep, nb1 = (size_t)nelem * hidden;
                 const size_t n2 = (size_t)nelem * d * hidden, nb2 = (size_t)nelem * d;
                 const size_t sizes[4] = {n1, nb1, n2, nb2};
                 DevBuf *ps[4] = {&h->w1, &h->b1, &h->w2, &h->b2};
                 for (int k = 0; k < 4; ++k) {
                     KFB_TRY(ps[k]->alloc(sizes[k] * sizeof(float), s));
                     KFB_TRY(zero(ps[k]->ptr, sizes[k] * sizeof(float), s));
                     KFB_TRY(h->mom[k].alloc(sizes[k] * sizeof(float), s));
                     KFB_TRY(h->var[k].alloc(sizes[k] * sizeof(float), s));
                     KFB_TRY(zero(h->mom[k].ptr, sizes[k] * sizeof(float), s));
                     KFB_TRY(zero(h->var[k].ptr, sizes[k] * sizeof(float), s));
                     KFB_TRY(h->grad[k].alloc(sizes[k] / nelem * sizeof(float), s));
                 }
                 KFB_TRY(h->w1b.alloc(n1 * sizeof(bf16), s));
                 KFB_TRY(h->w2b.alloc(n2 * sizeof(bf16), s));
                 KFB_TRY(h->w2tb.alloc(n2 * sizeof(bf16), s));
                 const long long R = 2 * ru8(max_pairs);
                 KFB_TRY(h->idx.alloc((size_t)R * sizeof(int), s));
                 KFB_TRY(h->xb.alloc((size_t)R * rep * sizeof(bf16), s));
                 KFB_TRY(h->xbt.alloc((size_t)R * rep * sizeof(bf16), s));
                 KFB_TRY(h->z1.alloc((size_t)R * hidden * sizeof(float), s));
                 KFB_TRY(h->hb.alloc((size_t)R * hidden * sizeof(bf16), s));
                 KFB_TRY(h->hbt.alloc((size_t)R * hidden * sizeof(bf16), s));
                 KFB_TRY(h->z2.alloc((size_t)R * d * sizeof(float), s));
                 KFB_TRY(h->dz2.alloc((size_t)R * d * sizeof(bf16), s));
                 KFB_TRY(h->dz2t.alloc((size_t)R * d * sizeof(bf16), s));
                 KFB_TRY(h->dz1t.alloc((size_t)R * hidden * sizeof(bf16), s));
                 KFB_TRY(h->loss.alloc(sizeof(double), s));
                 KFB_TRY(h->err.alloc(2 * sizeof(int), s));
                 KFB_CUDA_TRY(cudaStreamSynchronize(s));
                 return KFB_OK;
             }()) != KFB_OK)
            return fail(st);
        *out = h;
        return KFB_OK;
    });
}

void kfb_cosmlp_destroy(kfb_cosmlp *h) {
    if (!h) return;
    cudaDeviceSynchronize();
    delete h;
}

kfb_status kfb_cosmlp_params(kfb_cosmlp *h, float **w1, float **b1, float **w2, float **b2) {
    KFB_TRY(check_cosmlp(h));
    if (w1) *w1 = h->w1.as<float>();
    if (b1) *b1 = h->b1.as<float>();
    if (w2) *w2 = h->w2.as<float>();
    if (b2) *b2 = h->b2.as<float>();
    return KFB_OK;
}

kfb_status kfb_cosmlp_grads(kfb_cosmlp *h, float **w1, float **b1, float **w2, float **b2) {
    KFB_TRY(check_cosmlp(h));
    if (w1) *w1 = h->grad[0].as<float>();
    if (b1) *b1 = h->grad[1].as<float>();
    if (w2) *w2 = h->grad[2].as<float>();
    if (b2) *b2 = h->grad[3].as<float>();
    return KFB_OK;
}

kfb_status kfb_cosmlp_sync(kfb_cosmlp *h, int reset_optimizer, void *stream) {
    KFB_TRY(check_cosmlp(h));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int H = h->hidden, D = h->d, rep = h->rep;
    for (int e = 0; e < h->nelem; ++e) {
        to_bf16_kernel<<<nblk((long long)H * rep, 1024), 256, 0, s>>>(
            h->w1.as<float>() + (size_t)e * H * rep, H, rep, h->w1b.as<bf16>() + (size_t)e * H * rep,
            nullptr);
        to_bf16_kernel<<<nblk((long long)D * H, 1024), 256, 0, s>>>(
            h->w2.as<float>() + (size_t)e * D * H, D, H, h->w2b.as<bf16>() + (size_t)e * D * H,
            nullptr);
        KFB_CUDA_TRY(cudaGetLastError());
        KFB_TRY(transpose_bf16(h->w2b.as<bf16>() + (size_t)e * D * H, D, H,
                               h->w2tb.as<bf16>() + (size_t)e * H * D, D, nullptr, s));
    }
    if (reset_optimizer) {
        const size_t sizes[4] = {(size_t)h->nelem * H * rep, (size_t)h->nelem * H,
                                 (size_t)h->nelem * D * H, (size_t)h->nelem * D};
        for (int k = 0; k < 4; ++k) {
            KFB_TRY(zero(h->mom[k].ptr, sizes[k] * sizeof(float), s));
            KFB_TRY(zero(h->var[k].ptr, sizes[k] * sizeof(float), s));
        }
        std::fill(h->steps.begin(), h->steps.end(), 0);
    }
    return KFB_OK;
}

kfb_status kfb_cosmlp_optimizer_state(kfb_cosmlp *h, float **m, float **v, int *steps) {
    KFB_TRY(check_cosmlp(h));
    for (int k = 0; k < 4; ++k) {
        if (m) m[k] = h->mom[k].as<float>();
        if (v) v[k] = h->var[k].as<float>();
    }
    if (steps)
        for (int e = 0; e < h->nelem; ++e) steps[e] = h->steps[e];
    return KFB_OK;
}

kfb_status kfb_cosmlp_set_steps(kfb_cosmlp *h, const int *steps) {
    KFB_TRY(check_cosmlp(h));
    if (!steps) return set_error(KFB_ERR_INVALID_ARG, "null pointer argument");
    for (int e = 0; e < h->nelem; ++e) h->steps[e] = steps[e];
    return KFB_OK;
}

kfb_status kfb_cosmlp_pair_step(kfb_cosmlp *h, int elem, const void *x, long long nrows,
                                kfb_dtype x_dtype, const int *pi, const int *pj,
                                const float *target, int npairs, float lr, int update,
                                double *loss, void *stream) {
    return guarded([&]() -> kfb_status {
        KFB_TRY(check_cosmlp(h));
        if (!x || !pi || !pj || !target)
            return set_error(KFB_ERR_INVALID_ARG, "null pointer argument");
        if (elem < 0 || elem >= h->nelem)
            return set_error(KFB_ERR_INVALID_ARG, "element %d out of range [0, %d)", elem,
                             h->nelem);
        if (nrows <= 0) return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
        if (npairs <= 0 || npairs > h->max_pairs)
            return set_error(KFB_ERR_INVALID_ARG, "npairs = %d outside [1, %d]", npairs,
                             h->max_pairs);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (x_dtype == KFB_F64)
            return cosmlp_step_t<double>(h, elem, static_cast<const double *>(x), nrows, pi, pj,
                                         target, npairs, lr, update, loss, s);
        return cosmlp_step_t<float>(h, elem, static_cast<const float *>(x), nrows, pi, pj, target,
                                    npairs, lr, update, loss, s);
    });
}

kfb_status kfb_cosmlp_features_elemental(kfb_cosmlp *h, const void *x, const int *q,
                                         const int *n, int nm, int ma, int rep, kfb_dtype x_dtype,
                                         float *z, void *stream) {
    return guarded([&]() -> kfb_status {
        KFB_TRY(check_cosmlp(h));
        if (!x || !q || !n || !z) return set_error(KFB_ERR_INVALID_ARG, "null pointer argument");
        if (nm <= 0 || ma <= 0) return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
        if (rep != h->rep)
            return set_error(KFB_ERR_INVALID_ARG, "rep = %d but the network takes %d", rep, h->rep);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        if (x_dtype == KFB_F64)
            return cosmlp_features_t<double>(h, static_cast<const double *>(x), q, n, nm, ma, z, s);
        return cosmlp_features_t<float>(h, static_cast<const float *>(x), q, n, nm, ma, z, s);
    });
}

}  // extern "C"
