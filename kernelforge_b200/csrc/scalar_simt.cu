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
#include "scalar_simt_kernels.cuh"

namespace kfb {

namespace {

using simt::pack_rows_kernel;
using simt::scalar_tile_kernel;
using simt::SK;
using simt::ST;

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
    const int Dp_ = (p.rep + SK - 1) / SK * SK;
    long long ntiles_ll = 0;
    const std::vector<SuperBlock> sbs =
        make_super_blocks(b1, bb, p.symmetric, ST, ST, (size_t)Dp_ * sizeof(T), ntiles_ll);
    if (ntiles_ll == 0) return KFB_OK;
    const int Dp = (p.rep + SK - 1) / SK * SK;
    DevBuf pa, na, ma, pb, nb, mb, dt;
    KFB_TRY((pack_set<Tin, T>(static_cast<const Tin *>(p.x1), b1, p.rep, Dp, pa, na, ma, s)));
    if (!p.symmetric)
        KFB_TRY((pack_set<Tin, T>(static_cast<const Tin *>(p.x2), b2, p.rep, Dp, pb, nb, mb, s)));
    KFB_TRY(expand_tiles(sbs, ntiles_ll, ST, ST, dt, s));
    const T coef = T(-1.0 / (2.0 * p.sigma * p.sigma));
    const DevBuf &PB = p.symmetric ? pa : pb, &NB = p.symmetric ? na : nb,
                 &MB = p.symmetric ? ma : mb;
    // grid-stride over tiles in launches of at most 2^31-1 blocks
    const size_t ntiles = (size_t)ntiles_ll;
    KernelTimer timer(s);
    timer.start();
    for (size_t off = 0; off < ntiles; off += (size_t)1 << 30) {
        const unsigned nb_ = (unsigned)std::min<size_t>(ntiles - off, (size_t)1 << 30);
        scalar_tile_kernel<T><<<nb_, simt::SIMT_THREADS, 0, s>>>(
            pa.as<T>(), PB.as<T>(), Dp, na.as<T>(), NB.as<T>(), ma.as<int>(), MB.as<int>(),
            dt.as<PairTile>() + off, coef, sink);
        KFB_CUDA_TRY(cudaGetLastError());
    }
    timer.stop();
    return KFB_OK;
}

}  // namespace

static int super_block_side(int tm, int tn, size_t row_bytes) {
    if (row_bytes == 0) return 1 << 30;  // unbounded: plain row-major order
    int dev = 0, l2 = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev) != cudaSuccess || l2 <= 0)
        l2 = 64 << 20;
    const size_t tile_bytes = (size_t)std::max(tm, tn) * row_bytes;
    return (int)std::max<size_t>(4, std::min<size_t>(64, (size_t)l2 / 2 / (2 * tile_bytes)));
}

// columns [first, end) of tile row ti inside super-block sb
__host__ __device__ inline void sb_row(const SuperBlock &sb, int ti, int &first, int &end) {
    first = sb.bj;
    if (sb.symmetric && ti > first) first = ti;
    end = sb.bj + sb.g < sb.ntj ? sb.bj + sb.g : sb.ntj;
}

std::vector<SuperBlock> make_super_blocks(const Buckets &a, const Buckets &b, bool symmetric,
                                          int tm, int tn, size_t row_bytes, long long &ntiles) {
    std::vector<SuperBlock> out;
    const int group = super_block_side(tm, tn, row_bytes);
    ntiles = 0;
    const int L = (int)a.labels.size();
    for (int l = 0; l < L; ++l) {
        const int sa = a.lab_start[l], ea = a.lab_start[l + 1];
        const int sb = b.lab_start[l], eb = b.lab_start[l + 1];
        if (ea <= sa || eb <= sb) continue;
        const int nti = (ea - sa + tm - 1) / tm, ntj = (eb - sb + tn - 1) / tn;
        for (int bi = 0; bi < nti; bi += group)
            for (int bj = symmetric ? bi : 0; bj < ntj; bj += group) {
                SuperBlock s{sa, ea, sb, eb, bi, bj, group, nti, ntj, symmetric ? 1 : 0, ntiles};
                long long cnt = 0;
                for (int ti = bi; ti < std::min(nti, bi + group); ++ti) {
                    int f, e;
                    sb_row(s, ti, f, e);
                    if (e > f) cnt += e - f;
                }
                if (cnt == 0) continue;
                out.push_back(s);
                ntiles += cnt;
            }
    }
    return out;
}

// Tile t of the list; `merge` consecutive column tiles of a super-block row
// form one tile (the last one of a row may be narrower: b_end stops at the
// row's own columns).  With merge > 1 the offsets of `sbs` count merged tiles
// (merge_offsets).
__global__ void expand_tiles_kernel(const SuperBlock *__restrict__ sbs, int nsb, long long ntiles,
                                    int tm, int tn, int merge, PairTile *__restrict__ out) {
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (t >= ntiles) return;
    int lo = 0, hi = nsb - 1;  // last super-block with offset <= t
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sbs[mid].offset <= t) lo = mid;
        else hi = mid - 1;
    }
    const SuperBlock sb = sbs[lo];
    long long local = t - sb.offset;
    const int ti_end = sb.bi + sb.g < sb.nti ? sb.bi + sb.g : sb.nti;
    for (int ti = sb.bi; ti < ti_end; ++ti) {
        int f, e;
        sb_row(sb, ti, f, e);
        const int c = e > f ? (e - f + merge - 1) / merge : 0;
        if (local < c) {
            const int tj = f + (int)local * merge;
            const int ncol = min(merge, e - tj);
            PairTile pt{};
            pt.a0 = sb.sa + ti * tm;
            pt.a_end = sb.ea;
            pt.b0 = sb.sb + tj * tn;
            pt.b_end = min(sb.eb, sb.sb + (tj + ncol) * tn);
            if (merge == 1) pt.b_end = sb.eb;
            pt.diag = (sb.symmetric && ti == tj) ? 1 : 0;
            out[t] = pt;
            return;
        }
        local -= c;
    }
}

long long merge_offsets(std::vector<SuperBlock> &sbs, int merge) {
    long long n = 0;
    for (SuperBlock &sb : sbs) {
        sb.offset = n;
        const int ti_end = std::min(sb.nti, sb.bi + sb.g);
        for (int ti = sb.bi; ti < ti_end; ++ti) {
            int f, e;
            sb_row(sb, ti, f, e);
            if (e > f) n += (e - f + merge - 1) / merge;
        }
    }
    return n;
}

kfb_status expand_tiles(const std::vector<SuperBlock> &sbs, long long ntiles, int tm, int tn,
                        DevBuf &tiles, cudaStream_t s, int merge) {
    KFB_TRY(tiles.alloc((size_t)std::max<long long>(ntiles, 1) * sizeof(PairTile), s));
    if (ntiles == 0) return KFB_OK;
    DevBuf dsb;
    KFB_TRY(upload(dsb, sbs, s));
    expand_tiles_kernel<<<(unsigned)((ntiles + 255) / 256), 256, 0, s>>>(
        dsb.as<SuperBlock>(), (int)sbs.size(), ntiles, tm, tn, merge, tiles.as<PairTile>());
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

std::vector<PairTile> make_pair_tiles(const Buckets &a, const Buckets &b, bool symmetric,
                                      int tm, int tn, size_t row_bytes, int merge) {
    std::vector<PairTile> out;
    long long n = 0;
    const std::vector<SuperBlock> sbs = make_super_blocks(a, b, symmetric, tm, tn, row_bytes, n);
    out.reserve((size_t)n);
    for (const SuperBlock &sb : sbs) {
        const int ti_end = std::min(sb.nti, sb.bi + sb.g);
        for (int ti = sb.bi; ti < ti_end; ++ti) {
            int f, e;
            sb_row(sb, ti, f, e);
            for (int tj = f; tj < e; tj += merge) {
                const int ncol = std::min(merge, e - tj);
                PairTile t{};
                t.a0 = sb.sa + ti * tm;
                t.a_end = sb.ea;
                t.b0 = sb.sb + tj * tn;
                t.b_end = merge == 1 ? sb.eb : std::min(sb.eb, sb.sb + (tj + ncol) * tn);
                t.diag = (sb.symmetric && ti == tj) ? 1 : 0;
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
