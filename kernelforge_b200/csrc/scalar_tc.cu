// Scalar FCHL19 local kernel on the sm_100a tensor cores (tcgen05 + TMEM + TMA).
//
// Same-label atoms are packed per label bucket (molecules in order), centred
// on the bucket mean and split into an fp16 pair x = hi + lo.  One persistent
// CTA per SM walks a list of 128 x 256 same-label tiles (two 128-column tiles
// of the L2-ordered plan merged, so each A slice feeds twice the MMA work):
//
//   warp 0      TMA producer: 64-wide K slices of A_hi, A_lo, B_hi, B_lo
//               (128B-swizzled) into a 2-stage shared-memory ring (96 KB each);
//   warp 1      MMA issuer: per K16 step, tcgen05.mma kind::f16
//               hi*hi + hi*lo + lo*hi into an FP32 accumulator in TMEM
//               (two accumulators, so the epilogue of tile t overlaps the
//               MMAs of tile t+1);
//   warp 2      TMEM allocator;
//   warps 4..11 epilogue (two per TMEM lane quadrant): tcgen05.ld of 32 x 32 accumulator blocks,
//               e_ij = exp2(c n_i + c n_j - 2c g_ij) with c = -log2(e)/(2 sigma^2),
//               reduction over (molecule a) x (molecule b) rectangles in
//               shared memory, one atomic add per rectangle into the output.
//
// Nothing of size N_atoms^2 leaves the SM.  Every mbarrier wait is bounded
// (about two seconds of %globaltimer); a wait that gives up raises an error
// flag that the host turns into KFB_ERR_TIMEOUT.
//
// Mathematics: kernel_gaussian / _symm / _symm_rfp, src/local_kernels.cpp:155-758.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <memory>
#include <cmath>
#include <mutex>

#include "kernels_common.cuh"
#include "scalar_plan.h"
#include "tc_common.cuh"

namespace kfb {

namespace {

using namespace tc;

constexpr int BM = 128;          // rows of A per tile (TMEM lanes)
constexpr int BN = 256;          // rows of B per tile (TMEM columns per accumulator)
constexpr int TN = 128;          // column tiles of the plan; a tile merges BN / TN of them
constexpr int MERGE = BN / TN;
constexpr int BK = 64;           // fp16 elements per K slice (128 bytes: one swizzle row)
constexpr int NSTAGE = 2;        // 96 KB per stage
constexpr int TILE_A_BYTES = BM * BK * 2;
constexpr int TILE_B_BYTES = BN * BK * 2;
constexpr int STAGE_BYTES = 2 * TILE_A_BYTES + 2 * TILE_B_BYTES;
constexpr int EPI_WARP0 = 4;
constexpr int NUM_EPI_WARPS = 8;              // two per TMEM lane quadrant
constexpr int NUM_THREADS = 32 * (EPI_WARP0 + NUM_EPI_WARPS);
constexpr int CHUNKS_PER_WARP = BN / 32 / (NUM_EPI_WARPS / 4);
constexpr int NACC = 2;                       // TMEM accumulator stages (4 measured no faster)
constexpr int TMEM_COLS = NACC * BN;
constexpr int SCR_LD = 33;
constexpr int SCR_FLOATS = 16 * SCR_LD;       // per epilogue warp: 16 column runs x 32 rows
constexpr int RUN_INTS = 4 * 33;              // rstart, cstart, rmol, cmol per warp

constexpr int OFF_STAGES = 0;
constexpr int OFF_SCR = OFF_STAGES + NSTAGE * STAGE_BYTES;
constexpr int OFF_RUNS = OFF_SCR + NUM_EPI_WARPS * SCR_FLOATS * 4;
constexpr int OFF_BARS = (OFF_RUNS + NUM_EPI_WARPS * RUN_INTS * 4 + 7) / 8 * 8;
constexpr int NBARS = 2 * NSTAGE + 2 * NACC + 1;  // full, empty, tmem_full, tmem_empty, mma_done
constexpr int OFF_TMEM = OFF_BARS + NBARS * 8;
constexpr int SMEM_BYTES = OFF_TMEM + 16;
constexpr int SMEM_ALLOC = SMEM_BYTES + 1024;  // slack for 1024-byte alignment
static_assert(SMEM_ALLOC <= 227 * 1024, "shared memory budget");

// Instruction descriptor, kind::f16: fp16 A and B (K-major), FP32 accumulator.
constexpr uint32_t IDESC = (1u << 4) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma_f16(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(IDESC), "r"(acc)
        : "memory");
}
// ------------------------------------------------------------------ kernel
// emit_pair in FP32 arithmetic (the rectangle sums are FP32 already)
__device__ __forceinline__ void emit_pair_f(const PairSink &s, int a, int b, float v, int diag) {
    v *= (float)s.scale;
    long long idx;
    if (s.mode == OUT_RECT) {
        idx = (long long)(a + s.row_off) * s.n + (b + s.col_off);
    } else {
        if (diag) {
            if (a > b) return;
        } else if (a == b) {
            v *= 2.f;
        }
        const long long r = a + s.row_off, c = b + s.col_off;
        if (s.layout == KFB_DENSE) {
            if (r != c) {
                if (s.out_f64) atomicAdd(static_cast<double *>(s.out) + c * s.n + r, (double)v);
                else atomicAdd(static_cast<float *>(s.out) + c * s.n + r, v);
            }
            idx = r * s.n + c;
        } else {
            idx = sym_index((kfb_layout)s.layout, s.n, r, c);
        }
    }
    if (s.out_f64) atomicAdd(static_cast<double *>(s.out) + idx, (double)v);
    else atomicAdd(static_cast<float *>(s.out) + idx, v);
}

__global__ void __launch_bounds__(NUM_THREADS, 1)
    scalar_tc_kernel(const __grid_constant__ CUtensorMap tm_a_hi,
                     const __grid_constant__ CUtensorMap tm_a_lo,
                     const __grid_constant__ CUtensorMap tm_b_hi,
                     const __grid_constant__ CUtensorMap tm_b_lo, int rep,
                     const float *__restrict__ nA, const float *__restrict__ nB,
                     const int *__restrict__ molA, const int *__restrict__ molB,
                     const PairTile *__restrict__ tiles, int ntiles, float m2c, PairSink sink,
                     int *err) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s_base = smem_u32(smem);
    const uint32_t bar0 = s_base + OFF_BARS;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (NSTAGE + s); };
    auto tfull_bar = [&](int a) { return bar0 + 8u * (2 * NSTAGE + a); };
    auto tempty_bar = [&](int a) { return bar0 + 8u * (2 * NSTAGE + NACC + a); };
    const uint32_t done_bar = bar0 + 8u * (2 * NSTAGE + 2 * NACC);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + OFF_TMEM);

    if (threadIdx.x == 0) {
        for (int s = 0; s < NSTAGE; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int a = 0; a < NACC; ++a) {
            mbar_init(tfull_bar(a), 1);
            mbar_init(tempty_bar(a), NUM_EPI_WARPS);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile(
            "tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                smem_u32(tmem_holder)),
            "r"(TMEM_COLS)
            : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_holder;
    const int nkb = (rep + BK - 1) / BK;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer
        if (lane == 0) {
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_a_hi)));
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_a_lo)));
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_b_hi)));
            asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&tm_b_lo)));
            int stage = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const PairTile tl = tiles[t];
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(empty_bar(stage), ph ^ 1u, err)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sa = s_base + OFF_STAGES + stage * STAGE_BYTES;
                    mbar_expect_tx(full_bar(stage), STAGE_BYTES);
                    tma_load_2d(sa, &tm_a_hi, kb * BK, tl.a0, full_bar(stage));
                    tma_load_2d(sa + TILE_A_BYTES, &tm_a_lo, kb * BK, tl.a0, full_bar(stage));
                    tma_load_2d(sa + 2 * TILE_A_BYTES, &tm_b_hi, kb * BK, tl.b0,
                                full_bar(stage));
                    tma_load_2d(sa + 2 * TILE_A_BYTES + TILE_B_BYTES, &tm_b_lo, kb * BK, tl.b0,
                                full_bar(stage));
                    if (++stage == NSTAGE) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            int stage = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                if (!mbar_wait(tempty_bar(acc), aph ^ 1u, err)) break;
                tc_fence_after();
                const uint32_t dtm = tmem_base + (uint32_t)(acc * BN);
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(full_bar(stage), ph, err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = s_base + OFF_STAGES + stage * STAGE_BYTES;
                    const int nks = min(BK / 16, (rep - kb * BK + 15) / 16);
                    for (int ks = 0; ks < nks; ++ks) {
                        const uint64_t ahi = sdesc(sa + ks * 32);
                        const uint64_t alo = sdesc(sa + TILE_A_BYTES + ks * 32);
                        const uint64_t bhi = sdesc(sa + 2 * TILE_A_BYTES + ks * 32);
                        const uint64_t blo = sdesc(sa + 2 * TILE_A_BYTES + TILE_B_BYTES + ks * 32);
                        umma_f16(dtm, ahi, bhi, (kb | ks) != 0 ? 1u : 0u);
                        umma_f16(dtm, ahi, blo, 1u);
                        umma_f16(dtm, alo, bhi, 1u);
                    }
                    umma_commit(empty_bar(stage));
                    if (++stage == NSTAGE) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(tfull_bar(acc));
                if (++acc == NACC) {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            // make sure every MMA issued has retired before TMEM is released
            umma_commit(done_bar);
            mbar_wait(done_bar, 0, err);
        }
    } else if (warp >= EPI_WARP0) {
        // ------------------------------------------------ epilogue
        // warp e handles TMEM lane quadrant q = warp % 4 (rows 32q..32q+31) and
        // column chunks [h * CHUNKS_PER_WARP, (h + 1) * CHUNKS_PER_WARP)
        const int e_id = warp - EPI_WARP0;
        const int q = warp & 3;
        const int h = e_id >> 2;
        float *scr = reinterpret_cast<float *>(smem + OFF_SCR) + e_id * SCR_FLOATS;
        int *runs = reinterpret_cast<int *>(smem + OFF_RUNS) + e_id * RUN_INTS;
        int *rstart = runs, *rmolr = runs + 66, *cmolr = runs + 99;   // 33 ints each
        const unsigned lt_mask = (1u << lane) - 1u;
        int acc = 0;
        uint32_t aph = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const PairTile tl = tiles[t];
            const int nra = min(BM, tl.a_end - tl.a0);
            const int nrb = min(BN, tl.b_end - tl.b0);
            // molecule runs of this warp's 32 rows
            const int row = q * 32 + lane;
            const bool rvalid = row < nra;
            const int rm = rvalid ? molA[tl.a0 + row] : -1;
            const float rn = rvalid ? nA[tl.a0 + row] : 0.f;
            const int rm_prev = __shfl_up_sync(0xffffffffu, rm, 1);
            const bool rst = rvalid && (lane == 0 || rm != rm_prev);
            const unsigned rmask = __ballot_sync(0xffffffffu, rst);
            const int nvr = __popc(__ballot_sync(0xffffffffu, rvalid));
            const int nr = __popc(rmask);
            if (rst) {
                rstart[__popc(rmask & lt_mask)] = lane;
                rmolr[__popc(rmask & lt_mask)] = rm;
            }
            if (lane == 0) rstart[nr] = nvr;

            const bool got = mbar_wait(tfull_bar(acc), aph, err);
            if (!__all_sync(0xffffffffu, got)) break;
            tc_fence_after();
            const uint32_t tbase = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * BN);
#pragma unroll 1
            for (int cc = 0; cc < CHUNKS_PER_WARP; ++cc) {
                const int c = h * CHUNKS_PER_WARP + cc;
                const int col = c * 32 + lane;
                const bool cvalid = col < nrb;
                const int cm = cvalid ? molB[tl.b0 + col] : -1;
                const float cn = cvalid ? nB[tl.b0 + col] : 0.f;
                const int cm_prev = __shfl_up_sync(0xffffffffu, cm, 1);
                const int cm_next = __shfl_down_sync(0xffffffffu, cm, 1);
                // column runs never cross the middle of the chunk, so each half
                // of 16 columns has at most 16 runs
                const bool cst = cvalid && (lane == 0 || lane == 16 || cm != cm_prev);
                const bool cend = cvalid && (lane == 15 || lane == 31 || cm != cm_next);
                const unsigned cmask = __ballot_sync(0xffffffffu, cst);
                const unsigned emask = __ballot_sync(0xffffffffu, cend);
                float v[32];
                tmem_ld32(tbase + (uint32_t)(c * 32), v);
                // only the first TN columns of a diagonal tile are its diagonal
                // block (the rest is the next, off-diagonal column tile); the
                // self pair (same packed row) of a diagonal block is exactly 1
                const int dg = (tl.diag && c * 32 < TN) ? 1 : 0;
                const bool has_self = dg && c == q;   // warp-uniform
#pragma unroll
                for (int hh = 0; hh < 2; ++hh) {
                    const unsigned hmask = hh ? 0xFFFF0000u : 0x0000FFFFu;
                    const unsigned cm_h = cmask & hmask;
                    const int nc = __popc(cm_h);
                    __syncwarp();
                    if (cst && (hmask & (1u << lane))) cmolr[__popc(cm_h & lt_mask)] = cm;
                    // per row: sums over each column run, kept in registers until
                    // the run ends (run boundaries are the same for every lane)
                    float run_sum = 0.f;
                    int k = 0;
                    if (has_self) {
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj) {
                            const int j = hh * 16 + jj;
                            const float cnj = __shfl_sync(0xffffffffu, cn, j);
                            float e = fast_exp2(fmaf(m2c, v[j], rn + cnj));
                            if (j == lane) e = 1.f;
                            run_sum += e;
                            if (emask & (1u << j)) {
                                scr[k * SCR_LD + lane] = run_sum;
                                ++k;
                                run_sum = 0.f;
                            }
                        }
                    } else {
#pragma unroll
                        for (int jj = 0; jj < 16; ++jj) {
                            const int j = hh * 16 + jj;
                            const float cnj = __shfl_sync(0xffffffffu, cn, j);
                            run_sum += fast_exp2(fmaf(m2c, v[j], rn + cnj));
                            if (emask & (1u << j)) {
                                scr[k * SCR_LD + lane] = run_sum;
                                ++k;
                                run_sum = 0.f;
                            }
                        }
                    }
                    __syncwarp();
                    // cross-row sums: one (row run, column run) rectangle per lane
                    const float inv_nc = 1.f / (float)max(nc, 1);
                    for (int p = lane; p < nr * nc; p += 32) {
                        const int ri = __float2int_rz(((float)p + 0.5f) * inv_nc);
                        const int ci = p - ri * nc;
                        const int r0 = rstart[ri], r1 = rstart[ri + 1];
                        const float *col_sums = scr + ci * SCR_LD;
                        // two independent partial sums: the loads overlap
                        float s0 = 0.f, s1 = 0.f;
                        int r = r0;
                        for (; r + 1 < r1; r += 2) {
                            s0 += col_sums[r];
                            s1 += col_sums[r + 1];
                        }
                        if (r < r1) s0 += col_sums[r];
                        emit_pair_f(sink, rmolr[ri], cmolr[ci], s0 + s1, dg);
                    }
                }
                __syncwarp();
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(tempty_bar(acc));
            if (++acc == NACC) {
                acc = 0;
                aph ^= 1u;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 2) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base),
                     "r"(TMEM_COLS)
                     : "memory");
    }
}

// Per-label mean of the set's active rows (FP64 partial sums, atomically
// combined): the centre each bucket is shifted to before the fp16 split.
// The rows of label l are [rs[l], re[l]) (the whole bucket, or the part of it
// that one chunk of molecules holds).
template <class Tin>
__global__ void label_mean_kernel(const Tin *__restrict__ x, const int *__restrict__ src,
                                  const int *__restrict__ rs, const int *__restrict__ re,
                                  int rep, int nsplit, double *__restrict__ mean) {
    const int l = blockIdx.z;
    const int s = rs[l], e = re[l];
    const int R = e - s;
    if (R <= 0) return;
    const int chunk = (R + nsplit - 1) / nsplit;
    const int r0 = s + blockIdx.y * chunk, r1 = min(e, r0 + chunk);
    const int k = blockIdx.x * 32 + (threadIdx.x & 31);
    const int w = threadIdx.x >> 5;
    __shared__ double part[8][32];
    double acc = 0.0;
    if (k < rep)
        for (int r = r0 + w; r < r1; r += 8) acc += (double)x[(size_t)src[r] * rep + k];
    part[w][threadIdx.x & 31] = acc;
    __syncthreads();
    if (w == 0 && k < rep) {
        double t = 0.0;
        for (int i = 0; i < 8; ++i) t += part[i][threadIdx.x];
        atomicAdd(&mean[(size_t)l * rep + k], t / (double)R);
    }
}

// Packed split rows: v = x - mean(label); hi = fp16(v); lo = fp16(v - hi);
// norm = c * ||v||^2 (FP64 sum, stored as float).  Rows rows[i] for i < nrows
// (rows null: rows 0 .. nrows-1).
template <class Tin>
__global__ void pack_split_kernel(const Tin *__restrict__ x, const int *__restrict__ src,
                                  const int *__restrict__ lab_start, int L, const int *rows,
                                  int nrows, int rep, int Dp, const double *__restrict__ mean,
                                  double c, __half *__restrict__ hi, __half *__restrict__ lo,
                                  float *__restrict__ norm) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= nrows) return;
    const int r = rows ? rows[i] : i;
    int l = 0;
    while (l + 1 < L && r >= lab_start[l + 1]) ++l;
    const Tin *xr = x + (size_t)src[r] * rep;
    const double *mu = mean + (size_t)l * rep;
    double s = 0.0;
    for (int k = lane; k < Dp; k += 32) {
        __half h = __float2half_rn(0.f), o = __float2half_rn(0.f);
        if (k < rep) {
            const double v = (double)xr[k] - mu[k];
            h = __float2half_rn((float)v);
            o = __float2half_rn((float)(v - (double)__half2float(h)));
            s += v * v;
        }
        hi[(size_t)r * Dp + k] = h;
        lo[(size_t)r * Dp + k] = o;
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) norm[r] = (float)(c * s);
}

// ---------------------------------------------------------------- host side
PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

kfb_status make_map(CUtensorMap *m, const __half *ptr, int rows, int Dp, int box_rows) {
    auto enc = get_encode();
    if (!enc) return set_error(KFB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    cuuint64_t gdim[2] = {(cuuint64_t)Dp, (cuuint64_t)std::max(rows, 1)};
    cuuint64_t gstride[1] = {(cuuint64_t)Dp * sizeof(__half)};
    cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 2, const_cast<__half *>(ptr), gdim,
                     gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(KFB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return KFB_OK;
}

struct SplitSet {
    DevBuf hi, lo, norm, mol, src, lab;
};

template <class Tin>
kfb_status pack_split(const Tin *x, const Buckets &bk, int rep, int Dp, const double *mean,
                      double c, SplitSet &o, cudaStream_t s) {
    const int R = bk.rows();
    const int L = (int)bk.labels.size();
    KFB_TRY(upload(o.src, bk.src, s));
    KFB_TRY(upload(o.mol, bk.mol, s));
    KFB_TRY(upload(o.lab, bk.lab_start, s));
    KFB_TRY(o.hi.alloc((size_t)std::max(R, 1) * Dp * sizeof(__half), s));
    KFB_TRY(o.lo.alloc((size_t)std::max(R, 1) * Dp * sizeof(__half), s));
    KFB_TRY(o.norm.alloc((size_t)std::max(R, 1) * sizeof(float), s));
    if (R > 0) {
        pack_split_kernel<Tin><<<(R + 7) / 8, 256, 0, s>>>(
            x, o.src.as<int>(), o.lab.as<int>(), L, nullptr, R, rep, Dp, mean, c,
            o.hi.as<__half>(), o.lo.as<__half>(), o.norm.as<float>());
        KFB_CUDA_TRY(cudaGetLastError());
    }
    return KFB_OK;
}

template <class Tin>
kfb_status run_tc(const ScalarProblem &p, const PairSink &sink, cudaStream_t s) {
    std::vector<int> labels = collect_labels(p.s1, p.symmetric ? nullptr : &p.s2);
    if (labels.empty()) return KFB_OK;
    TraceScope tr_all("scalar_tc", s);
    auto tr_plan = std::make_unique<TraceScope>("scalar_tc:plan", s);
    Buckets b1 = make_buckets(p.s1, labels);
    Buckets b2 = p.symmetric ? Buckets() : make_buckets(p.s2, labels);
    const Buckets &bb = p.symmetric ? b1 : b2;
    // packed rows: hi + lo fp16 halves of Dp columns
    const size_t packed_row_bytes = (size_t)((p.rep + 7) / 8 * 8) * 2 * sizeof(__half);
    long long ntiles_ll = 0;
    std::vector<SuperBlock> sbs =
        make_super_blocks(b1, bb, p.symmetric, BM, TN, packed_row_bytes, ntiles_ll);
    ntiles_ll = merge_offsets(sbs, MERGE);
    tr_plan.reset();
    auto tr_pack = std::make_unique<TraceScope>("scalar_tc:pack", s);
    if (ntiles_ll == 0) return KFB_OK;
    if (ntiles_ll > INT_MAX) return set_error(KFB_ERR_UNSUPPORTED, "too many tiles (%lld)", ntiles_ll);
    const int L = (int)labels.size();
    const int Dp = (p.rep + 7) / 8 * 8;
    const double log2e = 1.4426950408889634;
    const double c = -log2e / (2.0 * p.sigma * p.sigma);

    // per-label centre from set 1
    DevBuf mean;
    KFB_TRY(mean.alloc((size_t)L * p.rep * sizeof(double), s));
    KFB_TRY(zero(mean.ptr, (size_t)L * p.rep * sizeof(double), s));
    SplitSet A, B;
    {
        DevBuf src1, lab1;
        KFB_TRY(upload(src1, b1.src, s));
        KFB_TRY(upload(lab1, b1.lab_start, s));
        const int nsplit = 16;
        dim3 g((p.rep + 31) / 32, nsplit, L);
        label_mean_kernel<Tin><<<g, 256, 0, s>>>(static_cast<const Tin *>(p.x1), src1.as<int>(),
                                                 lab1.as<int>(), lab1.as<int>() + 1, p.rep,
                                                 nsplit, mean.as<double>());
        KFB_CUDA_TRY(cudaGetLastError());
    }
    KFB_TRY(pack_split<Tin>(static_cast<const Tin *>(p.x1), b1, p.rep, Dp, mean.as<double>(), c,
                            A, s));
    if (!p.symmetric)
        KFB_TRY(pack_split<Tin>(static_cast<const Tin *>(p.x2), b2, p.rep, Dp,
                                mean.as<double>(), c, B, s));
    const SplitSet &BB = p.symmetric ? A : B;

    CUtensorMap ma_hi, ma_lo, mb_hi, mb_lo;
    KFB_TRY(make_map(&ma_hi, A.hi.as<__half>(), b1.rows(), Dp, BM));
    KFB_TRY(make_map(&ma_lo, A.lo.as<__half>(), b1.rows(), Dp, BM));
    KFB_TRY(make_map(&mb_hi, BB.hi.as<__half>(), bb.rows(), Dp, BN));
    KFB_TRY(make_map(&mb_lo, BB.lo.as<__half>(), bb.rows(), Dp, BN));

    DevBuf dtiles, derr;
    KFB_TRY(expand_tiles(sbs, ntiles_ll, BM, TN, dtiles, s, MERGE));
    tr_pack.reset();
    TraceScope tr_kern("scalar_tc:kernel+wait", s);
    KFB_TRY(derr.alloc(sizeof(int), s));
    KFB_TRY(zero(derr.ptr, sizeof(int), s));

    static bool attr_set = false;
    if (!attr_set) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(scalar_tc_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_ALLOC));
        attr_set = true;
    }
    const int ntiles = (int)ntiles_ll;
    const int grid = std::min(ntiles, device_sm_count());
    KernelTimer timer(s);
    timer.start();
    scalar_tc_kernel<<<grid, NUM_THREADS, SMEM_ALLOC, s>>>(
        ma_hi, ma_lo, mb_hi, mb_lo, p.rep, A.norm.as<float>(), BB.norm.as<float>(),
        A.mol.as<int>(), BB.mol.as<int>(), dtiles.as<PairTile>(), ntiles, (float)(-2.0 * c),
        sink, derr.as<int>());
    KFB_CUDA_TRY(cudaGetLastError());
    timer.stop();
    int herr = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&herr, derr.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) return set_error(KFB_ERR_TIMEOUT, "tensor-core scalar kernel: a pipeline wait timed out");
    return KFB_OK;
}

// One non-blocking copy stream per device for the pipelined host input.
cudaStream_t h2d_stream() {
    static std::mutex mu;
    static cudaStream_t streams[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (!streams[dev] && cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking) != cudaSuccess) {
        (void)cudaGetLastError();
        streams[dev] = nullptr;
    }
    return streams[dev];
}

struct EventSet {
    std::vector<cudaEvent_t> ev;
    ~EventSet() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
    kfb_status create(int n) {
        ev.assign(n, nullptr);
        for (int i = 0; i < n; ++i)
            KFB_CUDA_TRY(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
        return KFB_OK;
    }
};

// Symmetric kernel from descriptors in host memory.  The copy of X runs in
// chunks of molecules on a copy stream while the tensor cores already work:
// a chunk's rows are centred and split as soon as it lands, and the tiles run
// in waves by the last chunk they need (rows are in molecule order inside a
// label bucket, so a tile's last row names its chunk).  A label is centred on
// the mean of its rows in the first chunk that has any.
template <class Tin>
kfb_status run_tc_from_host(const ScalarProblem &p, const Tin *xh, const PairSink &sink,
                            cudaStream_t s) {
    std::vector<int> labels = collect_labels(p.s1, nullptr);
    if (labels.empty()) return KFB_OK;
    TraceScope tr_all("scalar_tc_host", s);
    const int nm = p.s1.nm, ma = p.s1.ma, rep = p.rep;
    const size_t mol_elems = (size_t)ma * rep;
    cudaStream_t cs = h2d_stream();
    if (!cs) return set_error(KFB_ERR_CUDA, "could not create the copy stream");
    DevBuf xd;
    KFB_TRY(xd.alloc((size_t)nm * mol_elems * sizeof(Tin), s));
    const char *env = getenv("KFB_H2D_CHUNKS");
    const int C = std::max(1, std::min(env ? atoi(env) : 8, nm));
    std::vector<int> m0(C + 1);
    for (int c = 0; c <= C; ++c) m0[c] = (int)((long long)nm * c / C);
    EventSet evs;
    KFB_TRY(evs.create(C + 1));
    // the copies start once the buffer exists on s; chunk 0 goes first, the
    // plan is built while it runs, and the other chunks are queued after the
    // plan's small uploads (copies from pageable memory would otherwise wait
    // behind the whole of X in the copy engine)
    KFB_CUDA_TRY(cudaEventRecord(evs.ev[C], s));
    KFB_CUDA_TRY(cudaStreamWaitEvent(cs, evs.ev[C], 0));
    // on every way out (errors included) the copies issued so far are waited
    // for: s before it frees the device buffer, the host before the caller
    // may reuse the host buffer
    struct CopyGuard {
        cudaStream_t s;
        const std::vector<cudaEvent_t> &ev;
        int issued = 0;
        ~CopyGuard() {
            for (int i = 0; i < issued; ++i) {
                cudaStreamWaitEvent(s, ev[i], 0);
                cudaEventSynchronize(ev[i]);
            }
        }
    } guard{s, evs.ev};
    auto copy_chunk = [&](int c) -> kfb_status {
        const size_t off = (size_t)m0[c] * mol_elems;
        KFB_CUDA_TRY(cudaMemcpyAsync(xd.as<Tin>() + off, xh + off,
                                     (size_t)(m0[c + 1] - m0[c]) * mol_elems * sizeof(Tin),
                                     cudaMemcpyHostToDevice, cs));
        KFB_CUDA_TRY(cudaEventRecord(evs.ev[c], cs));
        guard.issued = c + 1;
        return KFB_OK;
    };
    KFB_TRY(copy_chunk(0));
    // plan (host, while the first chunk is copied)
    auto tr_plan = std::make_unique<TraceScope>("scalar_tc_host:plan", s);
    const Buckets b1 = make_buckets(p.s1, labels);
    const int L = (int)labels.size(), R = b1.rows();
    std::vector<int> chunk_of(nm);
    for (int c = 0; c < C; ++c)
        for (int m = m0[c]; m < m0[c + 1]; ++m) chunk_of[m] = c;
    // rows of each chunk; per chunk the row range of each label whose first
    // chunk it is (the rows its mean is taken over), empty otherwise
    std::vector<int> rows_all, rows_off(C + 1, 0), first(L, -1);
    std::vector<std::vector<int>> rows_c(C);
    std::vector<int> mrs((size_t)C * L, 0), mre((size_t)C * L, 0);
    for (int l = 0; l < L; ++l)
        for (int r = b1.lab_start[l]; r < b1.lab_start[l + 1];) {
            const int c = chunk_of[b1.mol[r]];
            int e = r;
            while (e < b1.lab_start[l + 1] && chunk_of[b1.mol[e]] == c) rows_c[c].push_back(e++);
            if (first[l] < 0) {
                first[l] = c;
                mrs[(size_t)c * L + l] = r;
                mre[(size_t)c * L + l] = e;
            }
            r = e;
        }
    for (int c = 0; c < C; ++c) {
        rows_off[c] = (int)rows_all.size();
        rows_all.insert(rows_all.end(), rows_c[c].begin(), rows_c[c].end());
    }
    rows_off[C] = (int)rows_all.size();
    // tiles, in waves by the chunk of their last row and column
    const size_t packed_row_bytes = (size_t)((rep + 7) / 8 * 8) * 2 * sizeof(__half);
    const std::vector<PairTile> tl =
        make_pair_tiles(b1, b1, true, BM, TN, packed_row_bytes, MERGE);
    if (tl.empty()) return KFB_OK;
    if (tl.size() > (size_t)INT_MAX) return set_error(KFB_ERR_UNSUPPORTED, "too many tiles");
    std::vector<int> wave(tl.size()), wstart(C + 1, 0);
    for (size_t t = 0; t < tl.size(); ++t) {
        const int ra = std::min(tl[t].a0 + BM, tl[t].a_end) - 1;
        const int rb = std::min(tl[t].b0 + BN, tl[t].b_end) - 1;
        wave[t] = std::max(chunk_of[b1.mol[ra]], chunk_of[b1.mol[rb]]);
        ++wstart[wave[t] + 1];
    }
    for (int c = 0; c < C; ++c) wstart[c + 1] += wstart[c];
    std::vector<PairTile> sorted(tl.size());
    {
        std::vector<int> pos(wstart.begin(), wstart.end() - 1);
        for (size_t t = 0; t < tl.size(); ++t) sorted[pos[wave[t]]++] = tl[t];
    }
    tr_plan.reset();
    const int Dp = (rep + 7) / 8 * 8;
    const double log2e = 1.4426950408889634;
    const double cexp = -log2e / (2.0 * p.sigma * p.sigma);
    SplitSet A;
    DevBuf mean, d_rows, d_mrs, d_mre, dtiles, derr;
    KFB_TRY(upload(A.src, b1.src, s));
    KFB_TRY(upload(A.mol, b1.mol, s));
    KFB_TRY(upload(A.lab, b1.lab_start, s));
    KFB_TRY(A.hi.alloc((size_t)std::max(R, 1) * Dp * sizeof(__half), s));
    KFB_TRY(A.lo.alloc((size_t)std::max(R, 1) * Dp * sizeof(__half), s));
    KFB_TRY(A.norm.alloc((size_t)std::max(R, 1) * sizeof(float), s));
    KFB_TRY(upload(d_rows, rows_all, s));
    KFB_TRY(upload(d_mrs, mrs, s));
    KFB_TRY(upload(d_mre, mre, s));
    KFB_TRY(upload(dtiles, sorted, s));
    KFB_TRY(mean.alloc((size_t)L * rep * sizeof(double), s));
    KFB_TRY(zero(mean.ptr, (size_t)L * rep * sizeof(double), s));
    KFB_TRY(derr.alloc(sizeof(int), s));
    KFB_TRY(zero(derr.ptr, sizeof(int), s));
    for (int c = 1; c < C; ++c) KFB_TRY(copy_chunk(c));
    CUtensorMap ma_hi, ma_lo, mb_hi, mb_lo;
    KFB_TRY(make_map(&ma_hi, A.hi.as<__half>(), R, Dp, BM));
    KFB_TRY(make_map(&ma_lo, A.lo.as<__half>(), R, Dp, BM));
    KFB_TRY(make_map(&mb_hi, A.hi.as<__half>(), R, Dp, BN));
    KFB_TRY(make_map(&mb_lo, A.lo.as<__half>(), R, Dp, BN));
    static bool attr_set = false;
    if (!attr_set) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(scalar_tc_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_ALLOC));
        attr_set = true;
    }
    KernelTimer timer(s);
    bool started = false;
    for (int c = 0; c < C; ++c) {
        KFB_CUDA_TRY(cudaStreamWaitEvent(s, evs.ev[c], 0));
        bool new_label = false;
        for (int l = 0; l < L; ++l) new_label |= first[l] == c;
        if (new_label) {
            const int nsplit = 16;
            dim3 g((rep + 31) / 32, nsplit, L);
            label_mean_kernel<Tin><<<g, 256, 0, s>>>(xd.as<Tin>(), A.src.as<int>(),
                                                     d_mrs.as<int>() + (size_t)c * L,
                                                     d_mre.as<int>() + (size_t)c * L, rep, nsplit,
                                                     mean.as<double>());
            KFB_CUDA_TRY(cudaGetLastError());
        }
        const int nr = rows_off[c + 1] - rows_off[c];
        if (nr > 0) {
            pack_split_kernel<Tin><<<(nr + 7) / 8, 256, 0, s>>>(
                xd.as<Tin>(), A.src.as<int>(), A.lab.as<int>(), L, d_rows.as<int>() + rows_off[c],
                nr, rep, Dp, mean.as<double>(), cexp, A.hi.as<__half>(), A.lo.as<__half>(),
                A.norm.as<float>());
            KFB_CUDA_TRY(cudaGetLastError());
        }
        const int nt = wstart[c + 1] - wstart[c];
        if (nt == 0) continue;
        if (!started) {
            timer.start();
            started = true;
        }
        const int grid = std::min(nt, device_sm_count());
        scalar_tc_kernel<<<grid, NUM_THREADS, SMEM_ALLOC, s>>>(
            ma_hi, ma_lo, mb_hi, mb_lo, rep, A.norm.as<float>(), A.norm.as<float>(),
            A.mol.as<int>(), A.mol.as<int>(), dtiles.as<PairTile>() + wstart[c], nt,
            (float)(-2.0 * cexp), sink, derr.as<int>());
        KFB_CUDA_TRY(cudaGetLastError());
    }
    timer.stop();
    int herr = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&herr, derr.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) return set_error(KFB_ERR_TIMEOUT, "tensor-core scalar kernel: a pipeline wait timed out");
    return KFB_OK;
}

}  // namespace

kfb_status scalar_tc_from_host(const ScalarProblem &p, const void *x_host, const PairSink &sink,
                               cudaStream_t s) {
    if (!device_is_sm100())
        return set_error(KFB_ERR_UNSUPPORTED,
                         "the split-fp16 tensor-core path needs an sm_100 (B200) device");
    if (!p.symmetric) return set_error(KFB_ERR_INVALID_ARG, "host input: symmetric kernel only");
    if (p.x_dt == KFB_F64) return run_tc_from_host<double>(p, static_cast<const double *>(x_host), sink, s);
    return run_tc_from_host<float>(p, static_cast<const float *>(x_host), sink, s);
}

kfb_status scalar_tc(const ScalarProblem &p, const PairSink &sink, cudaStream_t s) {
    if (!device_is_sm100())
        return set_error(KFB_ERR_UNSUPPORTED,
                         "the split-fp16 tensor-core path needs an sm_100 (B200) device");
    if (p.x_dt == KFB_F64) return run_tc<double>(p, sink, s);
    return run_tc<float>(p, sink, s);
}

}  // namespace kfb
