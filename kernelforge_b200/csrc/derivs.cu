// Jacobian and Hessian FCHL19 local kernels on CUDA cores (FP64 / FP32).
//
// Jacobian (+dK/dR of the "inner" set, src/local_kernels.cpp:791-974):
//   K[o, off_m + c] = sum_{j in m} v_{o,j} . J_j[:, c],
//   v_{o,j} = sum_{i in o, q_i = q_j} (e_ij / sigma^2) (x_i - x_j)
// The v rows are formed first (one warp per (o, j)), then contracted with the
// Jacobians by a grouped GEMM, one problem per inner molecule m.  This costs
// 2 rep 3 n_m per (o, j) instead of per atom pair.  The transposed Jacobian
// (src/local_kernels.cpp:991-1166) is the same contraction with the roles of
// the sets swapped, negated and written transposed.
//
// Hessian (src/local_kernels.cpp:1171-1419):
//   H_ab = sum_{i in a} J_i^T Y_i,
//   Y_i  = sum_{j in b, q_j = q_i} (w_ij J_j - w'_ij d_ij (J_j^T d_ij)^T),
//   d_ij = x_i - x_j, w = e/sigma^2, w' = e/sigma^4
// t_ij = J_j^T d_ij is formed once per atom pair (kernel 1), Y_i per
// (pair, i, 32-row slice of rep) (kernel 2) and H_ab = J_a^T Y by the grouped
// GEMM (kernel 3).
#include <algorithm>
#include <memory>

#include "derivs.h"
#include "kernels_common.cuh"
#include "tc_gemm.h"

namespace kfb {

namespace {

// ------------------------------------------------------------ grouped GEMM
constexpr int GT = 64, GK = 16;

template <class T>
__global__ void __launch_bounds__(256) gemm_grouped_kernel(const GemmProb *__restrict__ probs,
                                                           const GemmTile *__restrict__ tiles,
                                                           ElemSink sink) {
    __shared__ T As[GK][GT + 1];
    __shared__ T Bs[GK][GT + 1];
    const GemmTile tl = tiles[blockIdx.x];
    const GemmProb pb = probs[tl.prob];
    const T *A = static_cast<const T *>(pb.A);
    const T *B = static_cast<const T *>(pb.B);
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);
    for (int k0 = 0; k0 < pb.K; k0 += GK) {
        if (pb.transA) {
            const int k = tid >> 4, m = (tid & 15) * 4;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int mm = tl.m0 + m + u, kk = k0 + k;
                As[k][m + u] = (mm < pb.M && kk < pb.K) ? A[(size_t)kk * pb.lda + mm] : T(0);
            }
        } else {
            const int m = tid >> 2, k = (tid & 3) * 4;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int mm = tl.m0 + m, kk = k0 + k + u;
                As[k + u][m] = (mm < pb.M && kk < pb.K) ? A[(size_t)mm * pb.lda + kk] : T(0);
            }
        }
        {
            const int k = tid >> 4, n = (tid & 15) * 4;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int nn = tl.n0 + n + u, kk = k0 + k;
                Bs[k][n + u] = (nn < pb.N && kk < pb.K) ? B[(size_t)kk * pb.ldb + nn] : T(0);
            }
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            T a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][ty * 4 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int m = tl.m0 + ty * 4 + i, n = tl.n0 + tx * 4 + j;
            if (m < pb.M && n < pb.N)
                sink_store(sink, pb.row_off + m, pb.col_off + n, (double)acc[i][j] * pb.alpha,
                           pb.diag);
        }
}

// --------------------------------------------------------- Jacobian: v rows
// One warp per (outer molecule o in [o0, o0+no), inner active atom u):
//   V[(o - o0) * NU + u, :] = sum_{i in o, q_i = q_u} w_iu (x_i - x_u)
template <class T>
__global__ void jac_v_kernel(const T *__restrict__ xo, const int *__restrict__ qo,
                             const int *__restrict__ no, int mao, int o0, int nout,
                             const T *__restrict__ xi, const int *__restrict__ u_src,
                             const int *__restrict__ u_lab, int NU, int rep, T c2, T is2,
                             T *__restrict__ V) {
    extern __shared__ unsigned char wsm_raw[];
    T *wsm = reinterpret_cast<T *>(wsm_raw);
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    if (gw >= (long long)nout * NU) return;
    const int ol = (int)(gw / NU), u = (int)(gw - (long long)ol * NU);
    const int o = o0 + ol;
    T *w = wsm + wib * mao;
    const T *xu = xi + (size_t)u_src[u] * rep;
    const int lab = u_lab[u];
    const int na = min(max(no[o], 0), mao);
    for (int i = 0; i < na; ++i) {
        T wi = T(0);
        if (qo[(size_t)o * mao + i] == lab) {
            const T *xa = xo + ((size_t)o * mao + i) * rep;
            T s = T(0);
            for (int k = lane; k < rep; k += 32) {
                const T d = xa[k] - xu[k];
                s = fma(d, d, s);
            }
            for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
            wi = kexp<T>(c2 * s) * is2;
        }
        if (lane == 0) w[i] = wi;
    }
    __syncwarp();
    T *vrow = V + ((size_t)ol * NU + u) * rep;
    for (int k = lane; k < rep; k += 32) {
        const T xuk = xu[k];
        T acc = T(0);
        for (int i = 0; i < na; ++i) {
            const T wi = w[i];
            if (wi != T(0)) acc = fma(wi, xo[((size_t)o * mao + i) * rep + k] - xuk, acc);
        }
        vrow[k] = acc;
    }
}

// ------------------------------------------------------- Hessian kernel 1
// Block per (pair p, atom i of a): for each same-label j of b,
//   W[p,i,j] = e/sigma^2, W2[p,i,j] = e/sigma^4, Tt[p,i,j,:] = J_j^T (x_i - x_j)
template <class T>
__global__ void hess_t_kernel(const HessPair *__restrict__ pairs, const T *__restrict__ x1,
                              const T *__restrict__ x2, const T *__restrict__ dx2,
                              const int *__restrict__ q1, const int *__restrict__ q2, int ma1,
                              int ma2, int rep, T c2, T is2, T is4, T *__restrict__ W,
                              T *__restrict__ W2, T *__restrict__ Tt) {
    extern __shared__ unsigned char hsm_raw[];
    T *d = reinterpret_cast<T *>(hsm_raw);  // rep
    __shared__ T red[32];
    const HessPair pr = pairs[blockIdx.y];
    const int i = blockIdx.x;
    if (i >= pr.na) return;
    const int ld2 = 3 * ma2;
    const size_t wbase = ((size_t)blockIdx.y * ma1 + i) * ma2;
    const int qi = q1[(size_t)pr.a * ma1 + i];
    const T *xi = x1 + ((size_t)pr.a * ma1 + i) * rep;
    for (int j = 0; j < pr.nb; ++j) {
        if (q2[(size_t)pr.b * ma2 + j] != qi) {
            if (threadIdx.x == 0) {
                W[wbase + j] = T(0);
                W2[wbase + j] = T(0);
            }
            continue;
        }
        const T *xj = x2 + ((size_t)pr.b * ma2 + j) * rep;
        T s = T(0);
        for (int k = threadIdx.x; k < rep; k += blockDim.x) {
            const T dk = xi[k] - xj[k];
            d[k] = dk;
            s = fma(dk, dk, s);
        }
        for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x < 32) {
            T v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : T(0);
            for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
            if (threadIdx.x == 0) red[0] = v;
        }
        __syncthreads();
        const T e = kexp<T>(c2 * red[0]);
        if (threadIdx.x == 0) {
            W[wbase + j] = e * is2;
            W2[wbase + j] = e * is4;
        }
        const T *Jj = dx2 + ((size_t)pr.b * ma2 + j) * rep * (size_t)ld2;
        for (int c = threadIdx.x; c < 3 * pr.nb; c += blockDim.x) {
            T acc = T(0);
            for (int k = 0; k < rep; ++k) acc = fma(Jj[(size_t)k * ld2 + c], d[k], acc);
            Tt[(wbase + j) * ld2 + c] = acc;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------- Hessian kernel 2
// Block per (pair p, atom i, 32-row slice of rep); thread (k, c):
//   Y[p, i, k, c] = sum_j W[p,i,j] J_j[k,c] - W2[p,i,j] (x_i[k] - x_j[k]) Tt[p,i,j,c]
template <class T>
__global__ void hess_y_kernel(const HessPair *__restrict__ pairs, const T *__restrict__ x1,
                              const T *__restrict__ x2, const T *__restrict__ dx2, int ma1,
                              int ma2, int rep, const T *__restrict__ W,
                              const T *__restrict__ W2, const T *__restrict__ Tt,
                              T *__restrict__ Y, float *__restrict__ amax) {
    const HessPair pr = pairs[blockIdx.z];
    const int i = blockIdx.y;
    if (i >= pr.na) return;
    float vmax = 0.f;
    const int ld2 = 3 * ma2;
    const int ncol = 3 * pr.nb;
    const size_t wbase = ((size_t)blockIdx.z * ma1 + i) * ma2;
    const T *xi = x1 + ((size_t)pr.a * ma1 + i) * rep;
    T *Yi = Y + ((size_t)blockIdx.z * ma1 + i) * rep * (size_t)ld2;
    for (int idx = threadIdx.x; idx < 32 * ncol; idx += blockDim.x) {
        const int kl = idx / ncol, c = idx - kl * ncol;
        const int k = blockIdx.x * 32 + kl;
        if (k >= rep) continue;
        const T xik = xi[k];
        T acc = T(0);
        for (int j = 0; j < pr.nb; ++j) {
            const T wj = W[wbase + j];
            if (wj == T(0)) continue;
            const T jv = dx2[(((size_t)pr.b * ma2 + j) * rep + k) * ld2 + c];
            const T dk = xik - x2[((size_t)pr.b * ma2 + j) * rep + k];
            acc = fma(wj, jv, acc);
            acc = fma(-W2[wbase + j] * dk, Tt[(wbase + j) * ld2 + c], acc);
        }
        Yi[(size_t)k * ld2 + c] = acc;
        vmax = fmaxf(vmax, fabsf((float)acc));
    }
    if (amax) {
        // largest |entry| written, for the power-of-two scale of the fp16 split
        for (int o = 16; o; o >>= 1) vmax = fmaxf(vmax, __shfl_xor_sync(0xffffffffu, vmax, o));
        if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(amax), __float_as_int(vmax));
    }
}

template <class T>
kfb_status launch_gemm(const std::vector<GemmProb> &probs, const ElemSink &sink,
                       cudaStream_t s) {
    if (probs.empty()) return KFB_OK;
    std::vector<GemmTile> tiles;
    for (int p = 0; p < (int)probs.size(); ++p)
        for (int m0 = 0; m0 < probs[p].M; m0 += GT)
            for (int n0 = 0; n0 < probs[p].N; n0 += GT) tiles.push_back(GemmTile{p, m0, n0, 0});
    if (tiles.empty()) return KFB_OK;
    DevBuf dp, dt;
    KFB_TRY(upload(dp, probs, s));
    KFB_TRY(upload(dt, tiles, s));
    for (size_t off = 0; off < tiles.size(); off += (size_t)1 << 30) {
        const unsigned nb = (unsigned)std::min<size_t>(tiles.size() - off, (size_t)1 << 30);
        gemm_grouped_kernel<T><<<nb, 256, 0, s>>>(dp.as<GemmProb>(), dt.as<GemmTile>() + off,
                                                  sink);
        KFB_CUDA_TRY(cudaGetLastError());
    }
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
    if (NU == 0 || outer.v.nm == 0) return KFB_OK;
    DevBuf d_usrc, d_ulab, d_qo, d_no;
    KFB_TRY(upload(d_usrc, u_src, s));
    KFB_TRY(upload(d_ulab, u_lab, s));
    std::vector<int> qo(outer.v.q, outer.v.q + (size_t)outer.v.nm * outer.v.ma);
    std::vector<int> no(outer.v.n, outer.v.n + outer.v.nm);
    KFB_TRY(upload(d_qo, qo, s));
    KFB_TRY(upload(d_no, no, s));
    const size_t row_bytes = (size_t)NU * rep * (sizeof(T) + (tc ? 2 * sizeof(__half) : 0));
    int chunk = (int)std::max<size_t>(1, budget_bytes() / std::max<size_t>(row_bytes, 1));
    chunk = std::min(chunk, outer.v.nm);
    DevBuf V, vh, vl, jth, jtl;
    float jt_scale = 1.f;
    KFB_TRY(V.alloc((size_t)chunk * NU * rep * sizeof(T), s));
    const int ma_in = inner.v.ma;
    if (tc) {
        // inner Jacobians as K-major split rows: Jt[(m, c)][(j, k)]
        const size_t jt_elems = (size_t)inner.v.nm * 3 * ma_in * ma_in * rep;
        KFB_TRY(jth.alloc(jt_elems * sizeof(__half), s));
        KFB_TRY(jtl.alloc(jt_elems * sizeof(__half), s));
        std::vector<int> nin(inner.v.nm);
        for (int m = 0; m < inner.v.nm; ++m) nin[m] = inner.v.natoms(m);
        DevBuf d_nin;
        KFB_TRY(upload(d_nin, nin, s));
        KFB_TRY(transpose_split_dx<T>(static_cast<const T *>(inner.dx), inner.v.nm, ma_in, rep,
                                      d_nin.as<int>(), jth.as<__half>(), jtl.as<__half>(),
                                      &jt_scale, s));
        KFB_TRY(vh.alloc((size_t)chunk * NU * rep * sizeof(__half), s));
        KFB_TRY(vl.alloc((size_t)chunk * NU * rep * sizeof(__half), s));
    }
    const T c2 = T(-1.0 / (2.0 * sigma * sigma)), is2 = T(1.0 / (sigma * sigma));
    const int ld_in = 3 * inner.v.ma;
    for (int o0 = 0; o0 < outer.v.nm; o0 += chunk) {
        const int nout = std::min(chunk, outer.v.nm - o0);
        const long long nwarps = (long long)nout * NU;
        const int wpb = 8;
        jac_v_kernel<T><<<(unsigned)((nwarps + wpb - 1) / wpb), wpb * 32,
                          wpb * outer.v.ma * sizeof(T), s>>>(
            static_cast<const T *>(outer.x), d_qo.as<int>(), d_no.as<int>(), outer.v.ma, o0,
            nout, static_cast<const T *>(inner.x), d_usrc.as<int>(), d_ulab.as<int>(), NU, rep,
            c2, is2, V.as<T>());
        KFB_CUDA_TRY(cudaGetLastError());
        if (tc) {
            float v_scale = 1.f;
            KFB_TRY(split_rows<T>(V.as<T>(), (long long)nout * NU * rep, vh.as<__half>(),
                                  vl.as<__half>(), &v_scale, s));
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
template <class T>
kfb_status hessian_core(const DerivSet &s1, const DerivSet &s2, int rep, double sigma,
                        bool symmetric, bool tc, ElemSink sink, cudaStream_t s) {
    std::vector<int> off1, off2;
    deriv_offsets(s1.v, off1);
    deriv_offsets(s2.v, off2);
    std::vector<HessPair> pairs;
    for (int a = 0; a < s1.v.nm; ++a) {
        const int na = s1.v.natoms(a);
        if (na == 0) continue;
        for (int b = symmetric ? a : 0; b < s2.v.nm; ++b) {
            const int nb = s2.v.natoms(b);
            if (nb == 0) continue;
            pairs.push_back(HessPair{a, b, na, nb});
        }
    }
    if (pairs.empty()) return KFB_OK;
    std::vector<int> q1(s1.v.q, s1.v.q + (size_t)s1.v.nm * s1.v.ma);
    std::vector<int> q2(s2.v.q, s2.v.q + (size_t)s2.v.nm * s2.v.ma);
    DevBuf d_q1, d_q2;
    KFB_TRY(upload(d_q1, q1, s));
    KFB_TRY(upload(d_q2, q2, s));
    const int ma1 = s1.v.ma, ma2 = s2.v.ma, ld1 = 3 * ma1, ld2 = 3 * ma2;
    const size_t per_pair = ((size_t)ma1 * ma2 * (2 + ld2) + (size_t)ma1 * rep * ld2) * sizeof(T) +
                            (tc ? (size_t)ma1 * rep * ld2 * 2 * sizeof(__half) : 0);
    int batch = (int)std::max<size_t>(1, budget_bytes() / per_pair);
    batch = std::min<int>(batch, (int)pairs.size());
    batch = std::min(batch, 65535);
    DevBuf W, W2, Tt, Y, dpairs;
    KFB_TRY(W.alloc((size_t)batch * ma1 * ma2 * sizeof(T), s));
    KFB_TRY(W2.alloc((size_t)batch * ma1 * ma2 * sizeof(T), s));
    KFB_TRY(Tt.alloc((size_t)batch * ma1 * ma2 * ld2 * sizeof(T), s));
    KFB_TRY(Y.alloc((size_t)batch * ma1 * rep * ld2 * sizeof(T), s));
    KFB_TRY(dpairs.alloc((size_t)batch * sizeof(HessPair), s));
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
    for (size_t p0 = 0; p0 < pairs.size(); p0 += batch) {
        const int np = (int)std::min<size_t>(batch, pairs.size() - p0);
        KFB_CUDA_TRY(cudaMemcpyAsync(dpairs.ptr, pairs.data() + p0, np * sizeof(HessPair),
                                     cudaMemcpyHostToDevice, s));
        auto tr_t = std::make_unique<TraceScope>("hessian:t", s);
        hess_t_kernel<T><<<dim3(ma1, np), 128, rep * sizeof(T), s>>>(
            dpairs.as<HessPair>(), static_cast<const T *>(s1.x), static_cast<const T *>(s2.x),
            static_cast<const T *>(s2.dx), d_q1.as<int>(), d_q2.as<int>(), ma1, ma2, rep, c2,
            is2, is4, W.as<T>(), W2.as<T>(), Tt.as<T>());
        KFB_CUDA_TRY(cudaGetLastError());
        tr_t.reset();
        auto tr_y = std::make_unique<TraceScope>("hessian:y", s);
        if (tc) KFB_TRY(zero(yamax.ptr, sizeof(float), s));
        hess_y_kernel<T><<<dim3((rep + 31) / 32, ma1, np), 256, 0, s>>>(
            dpairs.as<HessPair>(), static_cast<const T *>(s1.x), static_cast<const T *>(s2.x),
            static_cast<const T *>(s2.dx), ma1, ma2, rep, W.as<T>(), W2.as<T>(), Tt.as<T>(),
            Y.as<T>(), tc ? yamax.as<float>() : nullptr);
        KFB_CUDA_TRY(cudaGetLastError());
        tr_y.reset();
        auto tr_g = std::make_unique<TraceScope>("hessian:split+gemm", s);
        if (tc) {
            float y_scale = 1.f;
            KFB_TRY(transpose_split_y<T>(Y.as<T>(), np, ma1, rep, ld2, yamax.as<float>(),
                                         yth.as<__half>(), ytl.as<__half>(), &y_scale, s));
            std::vector<TcProb> tprobs;
            tprobs.reserve(np);
            for (int k = 0; k < np; ++k) {
                const HessPair &pr = pairs[p0 + k];
                TcProb p{};
                p.a_row0 = pr.a * ld1;
                p.a_k0 = 0;
                p.b_row0 = k * ld2;
                p.b_k0 = 0;
                p.M = 3 * pr.na;
                p.N = 3 * pr.nb;
                p.K = pr.na * rep;
                p.row_off = off1[pr.a];
                p.col_off = off2[pr.b];
                p.diag = (symmetric && pr.a == pr.b) ? 1 : 0;
                p.alpha = 1.0 / ((double)jt_scale * (double)y_scale);
                tprobs.push_back(p);
            }
            TcOperand A, B;
            A.hi = jth.ptr;
            A.lo = jtl.ptr;
            A.rows = (long long)s1.v.nm * ld1;
            A.cols = (long long)ma1 * rep;
            B.hi = yth.ptr;
            B.lo = ytl.ptr;
            B.rows = (long long)np * ld2;
            B.cols = (long long)ma1 * rep;
            KFB_TRY(tc_gemm_grouped(A, B, 3, false, tprobs, sink, s));
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
