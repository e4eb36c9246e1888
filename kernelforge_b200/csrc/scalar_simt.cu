// Scalar FCHL19 local kernel on CUDA cores (FP64 or FP32): the plain GPU
// path.  Atoms are bucketed by label (one packed, zero-padded row per atom,
// molecules in order inside a bucket); each CTA computes one 64 x 64 tile of
// same-label atom pairs, forms e_ij = exp(-(n_i + n_j - 2 x_i.x_j) / 2 sigma^2)
// in registers and reduces the tile over (molecule a) x (molecule b)
// rectangles before one atomic add per rectangle.  No N_atoms^2 intermediate
// is written to global memory.
//
// Mathematics: kernel_gaussian / _symm / _symm_rfp, src/local_kernels.cpp:155-758.
#include <algorithm>

#include "kernels_common.cuh"
#include "scalar_plan.h"

namespace kfb {

namespace {

constexpr int ST = 64;    // tile edge (rows of A and of B)
constexpr int SK = 16;    // K chunk staged in shared memory
constexpr int SPAD = 1;

template <class Tin, class T>
__global__ void pack_rows_kernel(const Tin *__restrict__ x, const int *__restrict__ src, int R,
                                 int rep, int Dp, T *__restrict__ out, T *__restrict__ norm) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= R) return;
    const Tin *xr = x + (size_t)src[warp] * rep;
    T *orow = out + (size_t)warp * Dp;
    double s = 0.0;
    for (int k = lane; k < Dp; k += 32) {
        const double v = k < rep ? (double)xr[k] : 0.0;
        orow[k] = (T)v;
        s += v * v;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) norm[warp] = (T)s;
}

template <class T>
__global__ void __launch_bounds__(256) scalar_tile_kernel(
    const T *__restrict__ A, const T *__restrict__ B, int Dp, const T *__restrict__ nA,
    const T *__restrict__ nB, const int *__restrict__ molA, const int *__restrict__ molB,
    const PairTile *__restrict__ tiles, T coef, PairSink sink) {
    // the staging tiles of the K loop and the e_ij tile of the epilogue share
    // one shared-memory buffer
    constexpr int STAGE_ELEMS = 2 * SK * (ST + SPAD), E_ELEMS = ST * (ST + SPAD);
    __shared__ T smem_buf[STAGE_ELEMS > E_ELEMS ? STAGE_ELEMS : E_ELEMS];
    T (*As)[ST + SPAD] = reinterpret_cast<T (*)[ST + SPAD]>(smem_buf);
    T (*Bs)[ST + SPAD] = reinterpret_cast<T (*)[ST + SPAD]>(smem_buf + SK * (ST + SPAD));
    T (*E)[ST + SPAD] = reinterpret_cast<T (*)[ST + SPAD]>(smem_buf);
    __shared__ int rmol[ST], cmol[ST];
    __shared__ int rstart[ST + 1], cstart[ST + 1];
    __shared__ int nrun_r, nrun_c;

    const PairTile t = tiles[blockIdx.x];
    const int tid = threadIdx.x;
    const int tx = tid & 15, ty = tid >> 4;
    const int nra = min(ST, t.a_end - t.a0);
    const int nrb = min(ST, t.b_end - t.b0);

    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);

    const int lr = tid >> 2, lk = (tid & 3) * 4;  // loader: row, first k
    for (int k0 = 0; k0 < Dp; k0 += SK) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int k = k0 + lk + u;
            As[lk + u][lr] = (lr < nra && k < Dp) ? A[(size_t)(t.a0 + lr) * Dp + k] : T(0);
            Bs[lk + u][lr] = (lr < nrb && k < Dp) ? B[(size_t)(t.b0 + lr) * Dp + k] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < SK; ++kk) {
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

    // e_ij into shared memory (zero outside the valid rows / columns)
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int r = ty * 4 + i;
        const T ni = r < nra ? nA[t.a0 + r] : T(0);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int c = tx * 4 + j;
            T v = T(0);
            if (r < nra && c < nrb) {
                const T d2 = ni + nB[t.b0 + c] - T(2) * acc[i][j];
                v = kexp<T>(coef * d2);
            }
            E[r][c] = v;
        }
    }
    if (tid < ST) rmol[tid] = tid < nra ? molA[t.a0 + tid] : -1;
    else if (tid < 2 * ST) cmol[tid - ST] = (tid - ST) < nrb ? molB[t.b0 + tid - ST] : -1;
    __syncthreads();
    // molecule runs along rows and columns
    if (tid == 0) {
        int k = 0;
        for (int r = 0; r < nra; ++r)
            if (r == 0 || rmol[r] != rmol[r - 1]) rstart[k++] = r;
        rstart[k] = nra;
        nrun_r = k;
    } else if (tid == 32) {
        int k = 0;
        for (int c = 0; c < nrb; ++c)
            if (c == 0 || cmol[c] != cmol[c - 1]) cstart[k++] = c;
        cstart[k] = nrb;
        nrun_c = k;
    }
    __syncthreads();
    const int nr = nrun_r, nc = nrun_c;
    for (int p = tid; p < nr * nc; p += blockDim.x) {
        const int ri = p / nc, ci = p - ri * nc;
        const int r0 = rstart[ri], r1 = rstart[ri + 1];
        const int c0 = cstart[ci], c1 = cstart[ci + 1];
        T s = T(0);
        for (int r = r0; r < r1; ++r)
            for (int c = c0; c < c1; ++c) s += E[r][c];
        emit_pair(sink, rmol[r0], cmol[c0], (double)s, t.diag);
    }
}

template <class Tin, class T>
kfb_status pack_set(const Tin *x, const Buckets &bk, int rep, int Dp, DevBuf &packed,
                    DevBuf &norms, DevBuf &mol, cudaStream_t s) {
    const int R = bk.rows();
    DevBuf src;
    KFB_TRY(upload(src, bk.src, s));
    KFB_TRY(upload(mol, bk.mol, s));
    KFB_TRY(packed.alloc((size_t)std::max(R, 1) * Dp * sizeof(T), s));
    KFB_TRY(norms.alloc((size_t)std::max(R, 1) * sizeof(T), s));
    if (R > 0) {
        const int threads = 256, rows_per_block = threads / 32;
        pack_rows_kernel<Tin, T><<<(R + rows_per_block - 1) / rows_per_block, threads, 0, s>>>(
            x, src.as<int>(), R, rep, Dp, packed.as<T>(), norms.as<T>());
        KFB_CUDA_TRY(cudaGetLastError());
    }
    return KFB_OK;
}

template <class Tin, class T>
kfb_status run_simt(const ScalarProblem &p, const PairSink &sink, cudaStream_t s) {
    std::vector<int> labels = collect_labels(p.s1, p.symmetric ? nullptr : &p.s2);
    if (labels.empty()) return KFB_OK;
    Buckets b1 = make_buckets(p.s1, labels);
    Buckets b2 = p.symmetric ? Buckets() : make_buckets(p.s2, labels);
    const Buckets &bb = p.symmetric ? b1 : b2;
    std::vector<PairTile> tiles = make_pair_tiles(b1, bb, p.symmetric, ST, ST);
    if (tiles.empty()) return KFB_OK;
    const int Dp = (p.rep + SK - 1) / SK * SK;
    DevBuf pa, na, ma, pb, nb, mb, dt;
    KFB_TRY((pack_set<Tin, T>(static_cast<const Tin *>(p.x1), b1, p.rep, Dp, pa, na, ma, s)));
    if (!p.symmetric)
        KFB_TRY((pack_set<Tin, T>(static_cast<const Tin *>(p.x2), b2, p.rep, Dp, pb, nb, mb, s)));
    KFB_TRY(upload(dt, tiles, s));
    const T coef = T(-1.0 / (2.0 * p.sigma * p.sigma));
    const DevBuf &PB = p.symmetric ? pa : pb, &NB = p.symmetric ? na : nb,
                 &MB = p.symmetric ? ma : mb;
    // grid-stride over tiles in launches of at most 2^31-1 blocks
    const size_t ntiles = tiles.size();
    KernelTimer timer(s);
    timer.start();
    for (size_t off = 0; off < ntiles; off += (size_t)1 << 30) {
        const unsigned nb_ = (unsigned)std::min<size_t>(ntiles - off, (size_t)1 << 30);
        scalar_tile_kernel<T><<<nb_, 256, 0, s>>>(pa.as<T>(), PB.as<T>(), Dp, na.as<T>(),
                                                   NB.as<T>(), ma.as<int>(), MB.as<int>(),
                                                   dt.as<PairTile>() + off, coef, sink);
        KFB_CUDA_TRY(cudaGetLastError());
    }
    timer.stop();
    return KFB_OK;
}

}  // namespace

std::vector<PairTile> make_pair_tiles(const Buckets &a, const Buckets &b, bool symmetric,
                                      int tm, int tn) {
    std::vector<PairTile> out;
    const int L = (int)a.labels.size();
    for (int l = 0; l < L; ++l) {
        const int sa = a.lab_start[l], ea = a.lab_start[l + 1];
        const int sb = b.lab_start[l], eb = b.lab_start[l + 1];
        if (ea <= sa || eb <= sb) continue;
        for (int i0 = sa; i0 < ea; i0 += tm) {
            const int j_first = symmetric ? i0 : sb;
            for (int j0 = j_first; j0 < eb; j0 += tn) {
                PairTile t{};
                t.a0 = i0;
                t.a_end = ea;
                t.b0 = j0;
                t.b_end = eb;
                t.diag = (symmetric && j0 == i0) ? 1 : 0;
                out.push_back(t);
            }
        }
    }
    return out;
}

kfb_status scalar_simt(const ScalarProblem &p, kfb_precision prec, const PairSink &sink,
                       cudaStream_t s) {
    if (prec == KFB_PREC_FP64) {
        if (p.x_dt == KFB_F64) return run_simt<double, double>(p, sink, s);
        return run_simt<float, double>(p, sink, s);
    }
    if (p.x_dt == KFB_F64) return run_simt<double, float>(p, sink, s);
    return run_simt<float, float>(p, sink, s);
}

}  // namespace kfb
