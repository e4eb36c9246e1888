// Contracted energy / force prediction with the local FCHL19 kernels (the
// "J^T alpha" form of src/local_kernels.cpp:2821-3425: compute_alpha_desc
// :2821-2894, hessian_matvec :2895-3154, jacobian_t_matvec :3155-3262,
// full_matvec :3263-3425): predictions of a model
// trained on energies and forces without forming the (query x training) E+F
// kernel matrix.
//
// With d = x_i - x_j, e = exp(-|d|^2 / 2 sigma^2), w = e / sigma^2,
// w2 = e / sigma^4 over same-label pairs (i query, j training atom) and
// Ad_j = J_j alpha_F,b (compute_alpha_desc):
//   E_a     = sum_{i in a, j} alpha_E[b] e + w (d . Ad_j)
//   F_(a,c) = sum_{i in a} J_i[:, c] . g_i,
//   g_i     = sum_j w Ad_j + sum_j v_ij d,  v_ij = -w alpha_E[b] - w2 (d . Ad_j)
//           = W Ad + rowsum(V) x_i - V X2     (W_ij = w, V_ij = v_ij)
// Per label bucket: G = X1 X2^T and P = X1 Ad^T as FP64-class products on the
// int8 tensor cores (ozaki.h: 7 digit planes per operand, exact int32 level
// sums combined in FP64), one fused kernel for e, w, v, the energy sums and
// W, V (written over G, P), two more such products for g (contracting over the
// label's training atoms, in chunks of 65,536), and a contraction of g with
// each query atom's Jacobian.  Every product is oriented so that the rows of
// its first operand run along the output's contiguous dimension (coalesced
// epilogue stores).  Query rows are processed in chunks that keep the two
// (rows x training atoms) matrices within the workspace budget.

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <memory>
#include <vector>

#include "kfb_internal.h"
#include "ozaki.h"

namespace kfb {

namespace {

unsigned nblk(long long n, int t) { return (unsigned)std::max<long long>(1, (n + t - 1) / t); }

// Ad[b, j, :] = dX2[b, j] (rep x 3 n_b) . alpha[off_b : off_b + 3 n_b]; zero
// for padded atoms.  Block per (b, j), threads over k.
template <class Tin>
__global__ void alpha_desc_kernel(const Tin *__restrict__ dx2, const int *__restrict__ n2,
                                  const int *__restrict__ off2, int ma2, int rep,
                                  const double *__restrict__ alpha, double *__restrict__ ad) {
    const int b = blockIdx.y, j = blockIdx.x;
    const int nb = min(max(n2[b], 0), ma2);
    const int ld = 3 * ma2, nc = 3 * nb;
    const double *al = alpha + off2[b];
    double *out = ad + ((size_t)b * ma2 + j) * rep;
    const Tin *J = dx2 + ((size_t)b * ma2 + j) * rep * (size_t)ld;
    for (int k = threadIdx.x; k < rep; k += blockDim.x) {
        double acc = 0.0;
        if (j < nb)
            for (int c = 0; c < nc; ++c) acc = fma((double)J[(size_t)k * ld + c], al[c], acc);
        out[k] = acc;
    }
}

// out[r, :] = (double) src[idx[r], :] (rows of rep values), and |row|^2
template <class Tin>
__global__ void gather_f64_kernel(const Tin *__restrict__ src, const int *__restrict__ idx,
                                  int nrows, int rep, double *__restrict__ out,
                                  double *__restrict__ norm2) {
    const int r = blockIdx.x;
    if (r >= nrows) return;
    const Tin *row = src + (size_t)idx[r] * rep;
    double s = 0.0;
    for (int k = threadIdx.x; k < rep; k += blockDim.x) {
        const double v = (double)row[k];
        out[(size_t)r * rep + k] = v;
        s = fma(v, v, s);
    }
    __shared__ double red[32];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0 && norm2) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        norm2[r] = t;
    }
}

// sc[r] = x_r . Ad_r and aE[r] = alpha_E[mol[r]] (0 without alpha_E)
__global__ void train_scalars_kernel(const double *__restrict__ X, const double *__restrict__ Ad,
                                     const int *__restrict__ mol, const double *__restrict__ alpha_e,
                                     int nrows, int rep, double *__restrict__ sc,
                                     double *__restrict__ ae) {
    const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= nrows) return;
    double s = 0.0;
    if (Ad)
        for (int k = lane; k < rep; k += 32) s = fma(X[(size_t)r * rep + k], Ad[(size_t)r * rep + k], s);
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        sc[r] = s;
        ae[r] = alpha_e ? alpha_e[mol[r]] : 0.0;
    }
}

// One block per query row i of the chunk: the Gaussian weights of all
// training atoms j of the label, the energy sum of row i (added to its
// molecule), and with forces W[i, j] = w, V[i, j] = v_ij (over G, P) and
// rowsum(V)[i].
__global__ void pair_weights_kernel(double *__restrict__ G, double *__restrict__ P, int r2,
                                    const double *__restrict__ n1, const double *__restrict__ n2,
                                    const double *__restrict__ sc, const double *__restrict__ ae,
                                    const int *__restrict__ mol1, int with_ad, int with_f,
                                    double c, double is2, double is4, double *__restrict__ E,
                                    double *__restrict__ rowv) {
    const int i = blockIdx.x;
    double *Gi = G + (size_t)i * r2;
    double *Pi = P + (size_t)i * r2;
    const double ni = n1[i];
    double esum = 0.0, vsum = 0.0;
    for (int j = threadIdx.x; j < r2; j += blockDim.x) {
        const double d2 = fmax(ni + n2[j] - 2.0 * Gi[j], 0.0);
        const double e = exp(c * d2);
        const double w = e * is2;
        const double dad = with_ad ? Pi[j] - sc[j] : 0.0;
        esum += ae[j] * e + w * dad;
        if (with_f) {
            const double v = -w * ae[j] - e * is4 * dad;
            Gi[j] = w;
            Pi[j] = v;
            vsum += v;
        }
    }
    __shared__ double red[2][32];
    for (int o = 16; o; o >>= 1) {
        esum += __shfl_xor_sync(0xffffffffu, esum, o);
        vsum += __shfl_xor_sync(0xffffffffu, vsum, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = esum;
        red[1][threadIdx.x >> 5] = vsum;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double te = 0.0, tv = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            te += red[0][w];
            tv += red[1][w];
        }
        if (E) atomicAdd(E + mol1[i], te);
        if (rowv) rowv[i] = tv;
    }
}

// g[i, :] += rowv[i] x1[i, :]
__global__ void add_row_scaled_kernel(const double *__restrict__ X1, const double *__restrict__ rowv,
                                      int rows, int rep, double *__restrict__ g) {
    const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (e < (long long)rows * rep) g[e] += rowv[e / rep] * X1[e];
}

// F[off_a + c] += sum_k dX1[a, i, k, c] g[r, k] for the query rows r of the
// chunk (molecule a, atom i); threads over c (coalesced along dX1 rows).
template <class Tin>
__global__ void force_contract_kernel(const Tin *__restrict__ dx1, const int *__restrict__ idx1,
                                      const int *__restrict__ mol1, const int *__restrict__ n1,
                                      const int *__restrict__ off1, int ma1, int rep,
                                      const double *__restrict__ g, double *__restrict__ F) {
    const int r = blockIdx.x;
    const int flat = idx1[r], a = mol1[r], i = flat - a * ma1;
    const int na = min(max(n1[a], 0), ma1);
    const int ld = 3 * ma1, nc = 3 * na;
    const Tin *J = dx1 + ((size_t)a * ma1 + i) * rep * (size_t)ld;
    const double *gr = g + (size_t)r * rep;
    for (int c = threadIdx.x; c < nc; c += blockDim.x) {
        double acc = 0.0;
        for (int k = 0; k < rep; ++k) acc = fma((double)J[(size_t)k * ld + c], gr[k], acc);
        atomicAdd(F + off1[a] + c, acc);
    }
}

size_t workspace_budget() {
    const char *v = std::getenv("KFB_WORKSPACE_GB");
    double gb = v ? std::atof(v) : 4.0;
    if (!(gb > 0)) gb = 4.0;
    return (size_t)(gb * (1ull << 30));
}

// FP64-class products on the int8 tensor cores (ozaki.h): 7 digit planes per
// operand (about 48 significant bits), exact int32 level sums combined in FP64.
constexpr int MV_S = 7;
constexpr int MV_KMAX = 65536;   // K of one product (int32 level sums stay exact)

// Digit planes of one operand, the buffers grown on demand.
struct MvOperand {
    DevBuf d, e;
    OzSlices sl;
    kfb_status reserve(long long rows, int K, cudaStream_t s) {
        const int kp = oz_kp(std::max(K, 1));
        const size_t nd = (size_t)MV_S * (size_t)std::max<long long>(rows, 1) * kp;
        const size_t ne = (size_t)std::max<long long>(rows, 1) * sizeof(int);
        if (d.bytes < nd) {
            d.release();
            KFB_TRY(d.alloc(nd, s));
        }
        if (e.bytes < ne) {
            e.release();
            KFB_TRY(e.alloc(ne, s));
        }
        sl.d = d.as<int8_t>();
        sl.e = e.as<int>();
        sl.S = MV_S;
        sl.rows = rows;
        sl.kp = kp;
        return KFB_OK;
    }
    // rows of a row-major source (ld between rows)
    kfb_status rows_of(const double *src, long long rows, int K, long long ld, cudaStream_t s) {
        KFB_TRY(reserve(rows, K, s));
        return oz_slice_rows<double>(src, rows, K, ld, sl, s);
    }
    // rows of the transpose of a row-major source: row i = column i
    kfb_status cols_of(const double *src, long long rows, int K, long long ld, DevBuf &mx,
                       cudaStream_t s) {
        KFB_TRY(reserve(rows, K, s));
        if (mx.bytes < (size_t)rows * 8) {
            mx.release();
            KFB_TRY(mx.alloc((size_t)rows * 8, s));
        }
        return oz_slice_colmajor(src, rows, K, ld, sl, mx.as<unsigned long long>(), s);
    }
};

// C[j * ldc + i] (or +=) alpha sum_k A[i][k] B[j][k] for i < M (rows of A),
// j < N (rows of B): A's rows run along C's contiguous dimension, so the
// epilogue's stores are coalesced.
kfb_status mv_gemm(const OzSlices &A, const OzSlices &B, int M, int N, double *C, long long ldc,
                   double alpha, bool add, int *err, cudaStream_t s) {
    OzGen g;
    g.mode = OZ_GEN_RECT;
    g.M = M;
    g.N = N;
    OzEpi epi;
    epi.c = C;
    epi.ldr = 1;
    epi.ldc = ldc;
    epi.mode = add ? OZ_ADD : OZ_STORE;
    epi.alpha = alpha;
    return oz_gemm_gen(A, B, g, epi, err, s);
}

template <class Tin>
kfb_status matvec_t(const Tin *x1, const Tin *dx1, const Tin *x2, const double *ad,
                    const double *alpha_e, const SetView &s1, const SetView &s2, int rep,
                    double sigma, double *E, double *F, cudaStream_t s) {
    if (E) KFB_TRY(zero(E, (size_t)s1.nm * sizeof(double), s));
    std::vector<int> off1;
    const long long naq1 = deriv_offsets(s1, off1);
    if (F) KFB_TRY(zero(F, (size_t)std::max<long long>(naq1, 1) * sizeof(double), s));
    const std::vector<int> labels = collect_labels(s1, &s2);
    if (labels.empty()) return KFB_OK;
    if (!device_is_sm100())
        return set_error(KFB_ERR_UNSUPPORTED, "the contracted prediction needs an sm_100 (B200) device");
    const Buckets b1 = make_buckets(s1, labels), b2 = make_buckets(s2, labels);
    std::vector<int> n1v(s1.nm);
    for (int m = 0; m < s1.nm; ++m) n1v[m] = s1.natoms(m);
    DevBuf dn1, doff1, didx1, dmol1, didx2, dmol2, derr, mx;
    KFB_TRY(upload(dn1, n1v, s));
    KFB_TRY(upload(doff1, off1, s));
    KFB_TRY(upload(didx1, b1.src, s));
    KFB_TRY(upload(dmol1, b1.mol, s));
    KFB_TRY(upload(didx2, b2.src, s));
    KFB_TRY(upload(dmol2, b2.mol, s));
    // one pipeline-timeout flag for every tensor-core product of the call
    KFB_TRY(derr.alloc(sizeof(int), s));
    KFB_TRY(zero(derr.ptr, sizeof(int), s));
    int *err = derr.as<int>();
    const double c = -1.0 / (2.0 * sigma * sigma), is2 = 1.0 / (sigma * sigma), is4 = is2 * is2;
    const bool with_ad = ad != nullptr, with_f = F != nullptr;
    MvOperand X2s, Ads, X1s, Ms;
    for (int l = 0; l < (int)labels.size(); ++l) {
        const int sa = b1.lab_start[l], r1 = b1.lab_start[l + 1] - sa;
        const int sb = b2.lab_start[l], r2 = b2.lab_start[l + 1] - sb;
        if (r1 == 0 || r2 == 0) continue;
        // training side of the label: X2, |x|^2, Ad, x.Ad, alpha_E of its molecule
        DevBuf X2l, n2l, Adl, scl, ael;
        KFB_TRY(X2l.alloc((size_t)r2 * rep * sizeof(double), s));
        KFB_TRY(n2l.alloc((size_t)r2 * sizeof(double), s));
        KFB_TRY(scl.alloc((size_t)r2 * sizeof(double), s));
        KFB_TRY(ael.alloc((size_t)r2 * sizeof(double), s));
        gather_f64_kernel<Tin><<<r2, 128, 0, s>>>(x2, didx2.as<int>() + sb, r2, rep,
                                                  X2l.as<double>(), n2l.as<double>());
        if (with_ad) {
            KFB_TRY(Adl.alloc((size_t)r2 * rep * sizeof(double), s));
            gather_f64_kernel<double><<<r2, 128, 0, s>>>(ad, didx2.as<int>() + sb, r2, rep,
                                                         Adl.as<double>(), nullptr);
        }
        train_scalars_kernel<<<nblk(r2, 8), 256, 0, s>>>(
            X2l.as<double>(), with_ad ? Adl.as<double>() : nullptr, dmol2.as<int>() + sb,
            alpha_e, r2, rep, scl.as<double>(), ael.as<double>());
        KFB_CUDA_TRY(cudaGetLastError());
        // digit planes of the training rows (K = rep) and, for the force
        // products g = W Ad - V X2 (K = r2, in chunks of MV_KMAX), of their
        // transposes
        KFB_TRY(X2s.rows_of(X2l.as<double>(), r2, rep, rep, s));
        if (with_ad) KFB_TRY(Ads.rows_of(Adl.as<double>(), r2, rep, rep, s));
        const int nkc = (r2 + MV_KMAX - 1) / MV_KMAX;
        std::vector<std::unique_ptr<MvOperand>> X2t, Adt;
        if (with_f)
            for (int kc = 0; kc < nkc; ++kc) {
                const int k0 = kc * MV_KMAX, kn = std::min(MV_KMAX, r2 - k0);
                X2t.emplace_back(new MvOperand);
                KFB_TRY(X2t.back()->cols_of(X2l.as<double>() + (size_t)k0 * rep, rep, kn, rep,
                                            mx, s));
                if (with_ad) {
                    Adt.emplace_back(new MvOperand);
                    KFB_TRY(Adt.back()->cols_of(Adl.as<double>() + (size_t)k0 * rep, rep, kn,
                                                rep, mx, s));
                }
            }
        // query rows in chunks: G and P (r1c x r2 each), X1 and g (r1c x rep)
        const size_t per_row = ((size_t)2 * r2 + 2 * rep + 2) * sizeof(double) +
                               (size_t)MV_S * (std::min(r2, MV_KMAX) + rep + 64);
        const int chunk = (int)std::max<size_t>(1, std::min<size_t>(r1, workspace_budget() / per_row));
        DevBuf X1c, n1c, Gm, Pm, gm, rowv;
        KFB_TRY(X1c.alloc((size_t)chunk * rep * sizeof(double), s));
        KFB_TRY(n1c.alloc((size_t)chunk * sizeof(double), s));
        KFB_TRY(Gm.alloc((size_t)chunk * r2 * sizeof(double), s));
        KFB_TRY(Pm.alloc((size_t)chunk * r2 * sizeof(double), s));
        if (with_f) {
            KFB_TRY(gm.alloc((size_t)chunk * rep * sizeof(double), s));
            KFB_TRY(rowv.alloc((size_t)chunk * sizeof(double), s));
        }
        for (int q0 = 0; q0 < r1; q0 += chunk) {
            const int rc = std::min(chunk, r1 - q0);
            gather_f64_kernel<Tin><<<rc, 128, 0, s>>>(x1, didx1.as<int>() + sa + q0, rc, rep,
                                                      X1c.as<double>(), n1c.as<double>());
            KFB_CUDA_TRY(cudaGetLastError());
            KFB_TRY(X1s.rows_of(X1c.as<double>(), rc, rep, rep, s));
            // G (rc x r2 row-major) = X1 X2^T, P = X1 Ad^T
            KFB_TRY(mv_gemm(X2s.sl, X1s.sl, r2, rc, Gm.as<double>(), r2, 1.0, false, err, s));
            if (with_ad)
                KFB_TRY(mv_gemm(Ads.sl, X1s.sl, r2, rc, Pm.as<double>(), r2, 1.0, false, err, s));
            pair_weights_kernel<<<rc, 256, 0, s>>>(
                Gm.as<double>(), Pm.as<double>(), r2, n1c.as<double>(), n2l.as<double>(),
                scl.as<double>(), ael.as<double>(), dmol1.as<int>() + sa + q0, with_ad ? 1 : 0,
                with_f ? 1 : 0, c, is2, is4, E, with_f ? rowv.as<double>() : nullptr);
            KFB_CUDA_TRY(cudaGetLastError());
            if (!with_f) continue;
            // g = W Ad + rowsum(V) x1 - V X2 (rc x rep row-major), W over G and V over P
            if (with_ad) {
                for (int kc = 0; kc < nkc; ++kc) {
                    const int k0 = kc * MV_KMAX, kn = std::min(MV_KMAX, r2 - k0);
                    KFB_TRY(Ms.rows_of(Gm.as<double>() + k0, rc, kn, r2, s));
                    KFB_TRY(mv_gemm(Adt[kc]->sl, Ms.sl, rep, rc, gm.as<double>(), rep, 1.0,
                                    kc > 0, err, s));
                }
            } else {
                KFB_TRY(zero(gm.ptr, (size_t)rc * rep * sizeof(double), s));
            }
            add_row_scaled_kernel<<<nblk((long long)rc * rep, 256), 256, 0, s>>>(
                X1c.as<double>(), rowv.as<double>(), rc, rep, gm.as<double>());
            KFB_CUDA_TRY(cudaGetLastError());
            for (int kc = 0; kc < nkc; ++kc) {
                const int k0 = kc * MV_KMAX, kn = std::min(MV_KMAX, r2 - k0);
                KFB_TRY(Ms.rows_of(Pm.as<double>() + k0, rc, kn, r2, s));
                KFB_TRY(mv_gemm(X2t[kc]->sl, Ms.sl, rep, rc, gm.as<double>(), rep, -1.0, true,
                                err, s));
            }
            force_contract_kernel<Tin><<<rc, 128, 0, s>>>(
                dx1, didx1.as<int>() + sa + q0, dmol1.as<int>() + sa + q0, dn1.as<int>(),
                doff1.as<int>(), s1.ma, rep, gm.as<double>(), F);
            KFB_CUDA_TRY(cudaGetLastError());
        }
    }
    int herr = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr)
        return set_error(KFB_ERR_TIMEOUT, "contracted prediction: a tensor-core pipeline wait timed out");
    return KFB_OK;
}

template <class Tin>
kfb_status alpha_desc_t(const Tin *dx2, const SetView &s2, int rep, const double *alpha,
                        double *ad, cudaStream_t s) {
    std::vector<int> off2;
    deriv_offsets(s2, off2);
    std::vector<int> n2v(s2.nm);
    for (int m = 0; m < s2.nm; ++m) n2v[m] = s2.natoms(m);
    DevBuf dn2, doff2;
    KFB_TRY(upload(dn2, n2v, s));
    KFB_TRY(upload(doff2, off2, s));
    alpha_desc_kernel<Tin><<<dim3(s2.ma, s2.nm), 256, 0, s>>>(dx2, dn2.as<int>(), doff2.as<int>(),
                                                             s2.ma, rep, alpha, ad);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

}  // namespace

}  // namespace kfb

using namespace kfb;

extern "C" {

kfb_status kfb_local_alpha_desc(const void *dx2, const int32_t *q2, const int32_t *n2, int nm2,
                                int ma2, int rep, kfb_dtype x_dt, const double *alpha,
                                double *alpha_desc, void *stream) {
    (void)q2;  // the contraction does not depend on the labels
    if (!dx2 || !n2 || !alpha || !alpha_desc)
        return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (nm2 <= 0 || ma2 <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "dimensions must be positive");
    SetView v;
    v.n = n2;
    v.nm = nm2;
    v.ma = ma2;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (x_dt == KFB_F64)
        return alpha_desc_t<double>(static_cast<const double *>(dx2), v, rep, alpha, alpha_desc, s);
    return alpha_desc_t<float>(static_cast<const float *>(dx2), v, rep, alpha, alpha_desc, s);
}

kfb_status kfb_local_matvec(const void *x1, const void *dx1, const void *x2,
                            const double *alpha_desc, const double *alpha_e, const int32_t *q1,
                            const int32_t *q2, const int32_t *n1, const int32_t *n2, int nm1,
                            int nm2, int ma1, int ma2, int rep, double sigma, kfb_dtype x_dt,
                            double *e_out, double *f_out, void *stream) {
    if (!x1 || !x2 || !q1 || !q2 || !n1 || !n2)
        return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (nm1 <= 0 || nm2 <= 0 || ma1 <= 0 || ma2 <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "dimensions must be positive");
    if (!(sigma > 0.0)) return set_error(KFB_ERR_INVALID_ARG, "sigma must be > 0");
    if (f_out && !dx1) return set_error(KFB_ERR_INVALID_ARG, "forces need dX1");
    if (!e_out && !f_out) return KFB_OK;
    SetView v1, v2;
    v1.q = q1;
    v1.n = n1;
    v1.nm = nm1;
    v1.ma = ma1;
    v2.q = q2;
    v2.n = n2;
    v2.nm = nm2;
    v2.ma = ma2;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (x_dt == KFB_F64)
        return matvec_t<double>(static_cast<const double *>(x1), static_cast<const double *>(dx1),
                                static_cast<const double *>(x2), alpha_desc, alpha_e, v1, v2, rep,
                                sigma, e_out, f_out, s);
    return matvec_t<float>(static_cast<const float *>(x1), static_cast<const float *>(dx1),
                           static_cast<const float *>(x2), alpha_desc, alpha_e, v1, v2, rep,
                           sigma, e_out, f_out, s);
}

}  // extern "C"
