// FP64-class products on the int8 tensor cores: slicing kernels and the
// tcgen05 kind::i8 GEMM (see ozaki.h for the scheme).
//
// Kernel roles (one persistent CTA per SM over a tile list, 384 threads):
//   warp 0      TMA producer: per 64-byte K slice, the S digit planes of the
//               A tile (128 rows) and of the B tile (BN = 128 rows for S <= 4,
//               else 64), 64-byte swizzle, into a shared-memory ring of 2-4
//               stages;
//   warp 1      MMA issuer: per K32 step, for every level L = 2 .. S+1 and every
//               digit pair p + q = L, tcgen05.mma kind::i8 (M=128, N=BN, K=32,
//               s32 accumulation) into level L's TMEM accumulator (BN columns
//               each, S accumulators side by side);
//   warp 2      TMEM allocator (512 columns);
//   warps 4..11 epilogue, two per TMEM lane quadrant (32-column chunks): load
//               the S int32 levels, combine them in FP64 (Horner in 2^-7),
//               release TMEM to the MMA issuer, then scale by 2^(e_a + e_b -
//               14) alpha and store / accumulate the FP64 outputs.
// Every mbarrier wait is bounded (%globaltimer); a wait that gives up raises
// the error flag instead of trapping.  No TMA multicast.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <mutex>

#include "ozaki.h"
#include "tc_common.cuh"

namespace kfb {

namespace {

using namespace tc;

constexpr int BM = OZ_BM, BK = OZ_BK;
constexpr int TILE_A = BM * BK;   // bytes per digit plane of an A tile
constexpr int EPI_WARP0 = 4, NUM_EPI_WARPS = 8;
constexpr int NUM_THREADS = 32 * (EPI_WARP0 + NUM_EPI_WARPS);
constexpr int TMEM_COLS = 512;

// S digit planes, BN output columns per tile (S BN <= 512 TMEM columns), as
// many pipeline stages (up to 4) as fit in 200 KB of shared memory.
template <int S>
struct OzCfg {
    static constexpr int BN = oz_bn(S);
    static constexpr int TILE_B = BN * BK;
    static constexpr int STAGE = S * (TILE_A + TILE_B);
    static constexpr int NSTAGE = (200 * 1024 / STAGE) < 4 ? (200 * 1024 / STAGE) : 4;
    static constexpr int OFF_BARS = NSTAGE * STAGE;
    static constexpr int NBARS = 2 * NSTAGE + 3;   // full, empty, tmem_full, tmem_empty, done
    static constexpr int OFF_TMEM = OFF_BARS + NBARS * 8;
    static constexpr int SMEM = OFF_TMEM + 16 + 1024;
    // instruction descriptor, kind::i8: signed A and B (K-major), s32 accumulator
    static constexpr uint32_t IDESC = (2u << 4) | (1u << 7) | (1u << 10) |
                                      ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
    static_assert(NSTAGE >= 2, "pipeline depth");
    static_assert(S * BN <= TMEM_COLS, "TMEM columns");
    static_assert(SMEM <= 227 * 1024, "shared memory budget");
};

// Shared-memory matrix descriptor: K-major, 64-byte swizzle (8-row groups
// 512 bytes apart), sm_100 version bit.
__device__ __forceinline__ uint64_t sdesc64(uint32_t saddr) {
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) |
           ((uint64_t)(512 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
}

__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// Column tiles of row tile ti in lower mode: the ones holding some j <= i.
__host__ __device__ __forceinline__ int lower_tiles(int ti, int ntc, int BN) {
    return min(ntc, ((ti + 1) * BM + BN - 1) / BN);
}

// Tile t of a generated tile set (see OzGen), BN columns per tile.
__host__ __device__ __forceinline__ OzTile gen_tile(const OzGen &g, int BN, long long ldr,
                                                    long long ldc, int t) {
    const int ntc = (g.N + BN - 1) / BN;
    int ti = 0, tj = t;
    if (g.mode == OZ_GEN_LOWER) {
        while (true) {
            const int cnt = lower_tiles(ti, ntc, BN);
            if (tj < cnt) break;
            tj -= cnt;
            ++ti;
        }
    } else {
        ti = t / ntc;
        tj = t - ti * ntc;
    }
    OzTile tl;
    tl.a0 = g.a_base + ti * BM;
    tl.b0 = g.b_base + tj * BN;
    tl.m = min(BM, g.M - ti * BM);
    tl.n = min(BN, g.N - tj * BN);
    tl.c_off = g.c_off + (long long)ti * BM * ldr + (long long)tj * BN * ldc;
    tl.lower = g.mode == OZ_GEN_LOWER ? 1 : 0;
    tl.lower_shift = g.b_base - g.a_base;
    return tl;
}

// 3-D tile load: box (x, y, z) of the tensor map into shared memory.
__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap *map, int x, int y,
                                            int z, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tmem_ld32_i(uint32_t taddr, int (&v)[32]) {
    float f[32];
    tmem_ld32(taddr, f);
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __float_as_int(f[i]);
}

template <int S>
__global__ void __launch_bounds__(NUM_THREADS, 1)
    oz_gemm_kernel(const __grid_constant__ CUtensorMap tm_a, const __grid_constant__ CUtensorMap tm_b,
                   long long a_rows, long long b_rows, int kp, const int *__restrict__ ea,
                   const int *__restrict__ eb, const OzTile *__restrict__ tiles, OzGen gen,
                   int ntiles, OzEpi epi, int *err) {
    using C = OzCfg<S>;
    constexpr int BN = C::BN, TILE_B = C::TILE_B, NSTAGE = C::NSTAGE;
    if (epi.skip && *(volatile const int *)epi.skip) return;   // block-uniform
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s_base = smem_u32(smem);
    const uint32_t bar0 = s_base + C::OFF_BARS;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (NSTAGE + s); };
    const uint32_t tfull_bar = bar0 + 8u * (2 * NSTAGE);
    const uint32_t tempty_bar = bar0 + 8u * (2 * NSTAGE + 1);
    const uint32_t done_bar = bar0 + 8u * (2 * NSTAGE + 2);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + C::OFF_TMEM);

    if (threadIdx.x == 0) {
        for (int s = 0; s < NSTAGE; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        mbar_init(tfull_bar, 1);
        mbar_init(tempty_bar, NUM_EPI_WARPS);
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_holder)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_holder;
    const int nkb = kp / BK;

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const OzTile tl = tiles ? tiles[t] : gen_tile(gen, BN, epi.ldr, epi.ldc, t);
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(empty_bar(stage), ph ^ 1u, err)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sa = s_base + stage * C::STAGE;
                    mbar_expect_tx(full_bar(stage), C::STAGE);
                    // all S planes of each operand tile in one 3-D box
                    tma_load_3d(sa, &tm_a, kb * BK, tl.a0, 0, full_bar(stage));
                    tma_load_3d(sa + S * TILE_A, &tm_b, kb * BK, tl.b0, 0, full_bar(stage));
                    if (++stage == NSTAGE) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                if (!mbar_wait(tempty_bar, aph ^ 1u, err)) break;
                tc_fence_after();
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!mbar_wait(full_bar(stage), ph, err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = s_base + stage * C::STAGE;
#pragma unroll
                    for (int ks = 0; ks < BK / 32; ++ks) {
#pragma unroll
                        for (int L = 2; L <= S + 1; ++L) {
                            const uint32_t dtm = tmem_base + (uint32_t)((L - 2) * BN);
#pragma unroll
                            for (int p = 1; p < L; ++p) {
                                const int q = L - p;
                                if (p > S || q > S) continue;
                                const uint64_t da = sdesc64(sa + (p - 1) * TILE_A + ks * 32);
                                const uint64_t db =
                                    sdesc64(sa + S * TILE_A + (q - 1) * TILE_B + ks * 32);
                                const bool first = kb == 0 && ks == 0 && p == 1;
                                umma_i8(dtm, da, db, C::IDESC, first ? 0u : 1u);
                            }
                        }
                    }
                    umma_commit(empty_bar(stage));
                    if (++stage == NSTAGE) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(tfull_bar);
                aph ^= 1u;
            }
            umma_commit(done_bar);
            mbar_wait(done_bar, 0, err);
        }
    } else if (warp >= EPI_WARP0) {
        // warp (q, h): TMEM lane quadrant q (tile rows 32 q ..), 32-column
        // chunks h, h + 2, ... of each level
        const int q = warp & 3;
        const int h = (warp - EPI_WARP0) >> 2;
        constexpr int NCH = BN / 64;
        uint32_t aph = 0;
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            const OzTile tl = tiles ? tiles[t] : gen_tile(gen, BN, epi.ldr, epi.ldc, t);
            const int i = q * 32 + lane;
            const bool got = mbar_wait(tfull_bar, aph, err);
            if (!__all_sync(0xffffffffu, got)) break;
            tc_fence_after();
#pragma unroll
            for (int ch = 0; ch < NCH; ++ch) {
                const int col0 = (h + 2 * ch) * 32;
                const uint32_t tb = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)col0;
                double acc[32];
                {
                    int v[32];
                    tmem_ld32_i(tb + (uint32_t)((S - 1) * BN), v);
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[j] = (double)v[j];
                }
#pragma unroll
                for (int l = S - 2; l >= 0; --l) {
                    int v[32];
                    tmem_ld32_i(tb + (uint32_t)(l * BN), v);
#pragma unroll
                    for (int j = 0; j < 32; ++j) acc[j] = fma(acc[j], 0.0078125, (double)v[j]);
                }
                if (ch == NCH - 1) {
                    // every level of this warp's chunks is in registers: hand
                    // TMEM back to the MMA issuer
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(tempty_bar);
                }
                if (i < tl.m) {
                    // columns col0 .. col0 + 31 of row i; nv of them are inside
                    // the tile (and on or below the diagonal in lower mode)
                    const int er = ea[tl.a0 + i] - 14;
                    double *crow = epi.c + tl.c_off + (long long)i * epi.ldr +
                                   (long long)col0 * epi.ldc;
                    const int *ebh = eb + tl.b0 + col0;
                    int nv = min(tl.n - col0, 32);
                    if (tl.lower) nv = min(nv, tl.a0 + i + tl.lower_shift - tl.b0 - col0 + 1);
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (j < nv) acc[j] = epi.alpha * oz_scale2(acc[j], er + ebh[j]);
                    if (epi.mode == OZ_ADD) {
                        // the loads of 16 old values first, then their stores: two
                        // memory latencies per chunk row instead of one per column
#pragma unroll
                        for (int hh = 0; hh < 32; hh += 16) {
                            double old[16];
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                if (hh + j < nv) old[j] = crow[(long long)(hh + j) * epi.ldc];
#pragma unroll
                            for (int j = 0; j < 16; ++j)
                                if (hh + j < nv)
                                    crow[(long long)(hh + j) * epi.ldc] = old[j] + acc[hh + j];
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < nv) crow[(long long)j * epi.ldc] = acc[j];
                    }
                }
            }
            aph ^= 1u;
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

// ------------------------------------------------------------------ slicing
// One warp per row of a row-major source; lanes over groups of 4 columns.
template <class T, int S>
__global__ void slice_rows_kernel(const T *__restrict__ src, long long rows, int K, long long ld,
                                  int kp, int8_t *__restrict__ d, int *__restrict__ e) {
    const long long r = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= rows) return;
    const T *row = src + r * ld;
    double m = 0.0;
    for (int k = lane; k < K; k += 32) m = fmax(m, fabs((double)row[k]));
    for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    const int ex = oz_row_exponent(m);
    if (lane == 0) e[r] = ex;
    const long long plane = rows * (long long)kp;
    for (int k0 = lane * 4; k0 < kp; k0 += 128) {
        int8_t dg[4][S];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int k = k0 + c;
            const double v = k < K ? ldexp((double)row[k], -ex) : 0.0;
            oz_digits<S>(v, dg[c]);
        }
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const uint32_t w = (uint32_t)(uint8_t)dg[0][s] | ((uint32_t)(uint8_t)dg[1][s] << 8) |
                               ((uint32_t)(uint8_t)dg[2][s] << 16) |
                               ((uint32_t)(uint8_t)dg[3][s] << 24);
            *reinterpret_cast<uint32_t *>(d + s * plane + r * kp + k0) = w;
        }
    }
}

// Column-major source: a block takes 32 rows, stages their K columns
// (coalesced along the rows) in shared memory, then one warp per row.
template <int S>
__global__ void slice_cols_kernel(const double *__restrict__ src, long long rows, int K,
                                  long long ld, int kp, int8_t *__restrict__ d,
                                  int *__restrict__ e) {
    extern __shared__ double tile[];   // [K][33]
    const long long r0 = (long long)blockIdx.x * 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    {
        // every load of the tile in flight at once (cp.async, 8 bytes each;
        // rows beyond the source are zero-filled)
        const long long r = r0 + lane;
        const bool ok = r < rows;
        const double *col0 = src + (ok ? r : 0);
        for (int k = warp; k < K; k += nw) {
            const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(tile + k * 33 + lane));
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d),
                         "l"(col0 + (long long)k * ld), "r"(ok ? 8 : 0)
                         : "memory");
        }
        asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncthreads();
    const long long plane = rows * (long long)kp;
    for (int rl = warp; rl < 32; rl += nw) {
        const long long r = r0 + rl;
        if (r >= rows) break;
        double m = 0.0;
        for (int k = lane; k < K; k += 32) m = fmax(m, fabs(tile[k * 33 + rl]));
        for (int o = 16; o; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        const int ex = oz_row_exponent(m);
        if (lane == 0) e[r] = ex;
        for (int k0 = lane * 4; k0 < kp; k0 += 128) {
            int8_t dg[4][S];
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const int k = k0 + c;
                const double v = k < K ? ldexp(tile[k * 33 + rl], -ex) : 0.0;
                oz_digits<S>(v, dg[c]);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint32_t w = (uint32_t)(uint8_t)dg[0][s] |
                                   ((uint32_t)(uint8_t)dg[1][s] << 8) |
                                   ((uint32_t)(uint8_t)dg[2][s] << 16) |
                                   ((uint32_t)(uint8_t)dg[3][s] << 24);
                *reinterpret_cast<uint32_t *>(d + s * plane + r * kp + k0) = w;
            }
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 oz_encoder() {
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

// The S digit planes of an operand as one 3-D int8 tensor (kp x rows x S),
// box 64 bytes x box_rows x S (all planes of a tile, stacked in shared
// memory as S tiles of box_rows x 64 bytes), 64-byte swizzle; rows beyond the
// operand read as zero.
kfb_status map_slices(CUtensorMap *m, const OzSlices &o, int box_rows) {
    auto enc = oz_encoder();
    if (!enc) return set_error(KFB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    const cuuint64_t rows = (cuuint64_t)std::max<long long>(o.rows, 1);
    cuuint64_t gdim[3] = {(cuuint64_t)o.kp, rows, (cuuint64_t)o.S};
    cuuint64_t gstride[2] = {(cuuint64_t)o.kp, (cuuint64_t)o.kp * rows};
    cuuint32_t box[3] = {(cuuint32_t)BK, (cuuint32_t)box_rows, (cuuint32_t)o.S};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, o.d, gdim, gstride, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return set_error(KFB_ERR_CUDA, "cuTensorMapEncodeTiled (digit planes) failed (%d)", (int)r);
    return KFB_OK;
}

template <int S>
kfb_status launch(const OzSlices &A, const OzSlices &B, const OzTile *tiles, const OzGen &gen,
                  int ntiles, const OzEpi &epi, int *err, cudaStream_t s) {
    using C = OzCfg<S>;
    CUtensorMap ta, tb;
    KFB_TRY(map_slices(&ta, A, BM));
    KFB_TRY(map_slices(&tb, B, C::BN));
    static bool attr[OZ_MAXS + 1] = {};
    if (!attr[S]) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(oz_gemm_kernel<S>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
        attr[S] = true;
    }
    const int grid = epi.one_tile_per_cta ? ntiles : std::min(ntiles, device_sm_count());
    oz_gemm_kernel<S><<<grid, NUM_THREADS, C::SMEM, s>>>(ta, tb, A.rows, B.rows, A.kp, A.e, B.e,
                                                         tiles, gen, ntiles, epi, err);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

template <class T>
kfb_status slice_rows_any(const T *src, long long rows, int K, long long ld, const OzSlices &o,
                          cudaStream_t s) {
    if (rows <= 0) return KFB_OK;
    const int wpb = 8;
    const unsigned g = (unsigned)((rows + wpb - 1) / wpb);
    switch (o.S) {
        case 2: slice_rows_kernel<T, 2><<<g, 32 * wpb, 0, s>>>(src, rows, K, ld, o.kp, o.d, o.e); break;
        case 3: slice_rows_kernel<T, 3><<<g, 32 * wpb, 0, s>>>(src, rows, K, ld, o.kp, o.d, o.e); break;
        case 4: slice_rows_kernel<T, 4><<<g, 32 * wpb, 0, s>>>(src, rows, K, ld, o.kp, o.d, o.e); break;
        case 5: slice_rows_kernel<T, 5><<<g, 32 * wpb, 0, s>>>(src, rows, K, ld, o.kp, o.d, o.e); break;
        case 6: slice_rows_kernel<T, 6><<<g, 32 * wpb, 0, s>>>(src, rows, K, ld, o.kp, o.d, o.e); break;
        case 7: slice_rows_kernel<T, 7><<<g, 32 * wpb, 0, s>>>(src, rows, K, ld, o.kp, o.d, o.e); break;
        default: return set_error(KFB_ERR_INVALID_ARG, "digit planes S=%d outside 2..%d", o.S, OZ_MAXS);
    }
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

}  // namespace

kfb_status oz_check(const OzSlices &o, int K) {
    if (o.S < 2 || o.S > OZ_MAXS)
        return set_error(KFB_ERR_INVALID_ARG, "digit planes S=%d outside 2..%d", o.S, OZ_MAXS);
    if (o.kp % OZ_BK != 0 || o.kp < K || o.kp > 65536)
        return set_error(KFB_ERR_INVALID_ARG, "digit-plane width %d (K=%d) must be a multiple of %d, "
                                              "at most 65536", o.kp, K, OZ_BK);
    return KFB_OK;
}

template <class T>
kfb_status oz_slice_rows(const T *src, long long rows, int K, long long ld, const OzSlices &out,
                         cudaStream_t s) {
    KFB_TRY(oz_check(out, K));
    return slice_rows_any<T>(src, rows, K, ld, out, s);
}
template kfb_status oz_slice_rows<double>(const double *, long long, int, long long,
                                          const OzSlices &, cudaStream_t);
template kfb_status oz_slice_rows<float>(const float *, long long, int, long long,
                                         const OzSlices &, cudaStream_t);

kfb_status oz_slice_cols(const double *src, long long rows, int K, long long ld,
                         const OzSlices &o, cudaStream_t s) {
    KFB_TRY(oz_check(o, K));
    if (rows <= 0) return KFB_OK;
    if (K > 512) return set_error(KFB_ERR_INVALID_ARG, "column-major slicing takes K <= 512");
    const unsigned g = (unsigned)((rows + 31) / 32);
    const size_t sm = (size_t)std::max(K, 1) * 33 * sizeof(double);
    switch (o.S) {
#define KFB_OZ_COLS(SS)                                                                       \
    case SS: {                                                                                \
        static bool a = false;                                                                \
        if (!a) {                                                                             \
            KFB_CUDA_TRY(cudaFuncSetAttribute(slice_cols_kernel<SS>,                           \
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                                              512 * 33 * (int)sizeof(double)));               \
            a = true;                                                                         \
        }                                                                                     \
        slice_cols_kernel<SS><<<g, 256, sm, s>>>(src, rows, K, ld, o.kp, o.d, o.e);           \
        break;                                                                                \
    }
        KFB_OZ_COLS(2)
        KFB_OZ_COLS(3)
        KFB_OZ_COLS(4)
        KFB_OZ_COLS(5)
        KFB_OZ_COLS(6)
        KFB_OZ_COLS(7)
#undef KFB_OZ_COLS
        default:
            return set_error(KFB_ERR_INVALID_ARG, "digit planes S=%d outside 2..%d", o.S, OZ_MAXS);
    }
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

namespace {

// mx[r] = max over k in this block's chunk of |src[k * ld + r]| (a column-major
// source read along r), combined across chunks by an atomic max on the bit
// pattern (non-negative doubles order like their 64-bit integers).
__global__ void colmajor_absmax_kernel(const double *__restrict__ src, long long rows, int K,
                                       long long ld, int kchunk,
                                       unsigned long long *__restrict__ mx) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    const int k0 = blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
    double m = 0.0;
    for (int k = k0; k < k1; ++k) m = fmax(m, fabs(src[(long long)k * ld + r]));
    atomicMax(mx + r, (unsigned long long)__double_as_longlong(m));
}

// Digits of a 32 (rows) x 32 (k) tile of a column-major source: staged in
// shared memory (read along the rows), written as 4 consecutive k per thread
// and plane (32-byte row segments).  Columns K .. kp-1 get zero digits.
template <int S>
__global__ void __launch_bounds__(256)
    colmajor_digits_kernel(const double *__restrict__ src, long long rows, int K, long long ld,
                           int kp, const unsigned long long *__restrict__ mx,
                           int8_t *__restrict__ d, int *__restrict__ e) {
    __shared__ double t[32][33];
    const long long r0 = (long long)blockIdx.x * 32;
    const int k0 = blockIdx.y * 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = warp; i < 32; i += 8) {
        const int k = k0 + i;
        const long long r = r0 + lane;
        t[i][lane] = (k < K && r < rows) ? src[(long long)k * ld + r] : 0.0;
    }
    __syncthreads();
    const int rr = warp * 4 + (lane >> 3), kk = (lane & 7) * 4;
    const long long r = r0 + rr;
    if (r >= rows) return;
    const int ex = oz_row_exponent(__longlong_as_double((long long)mx[r]));
    if (blockIdx.y == 0 && kk == 0) e[r] = ex;
    int8_t dg[4][S];
#pragma unroll
    for (int c = 0; c < 4; ++c) oz_digits<S>(ldexp(t[kk + c][rr], -ex), dg[c]);
    const long long plane = rows * (long long)kp;
#pragma unroll
    for (int sl = 0; sl < S; ++sl) {
        const uint32_t wv = (uint32_t)(uint8_t)dg[0][sl] | ((uint32_t)(uint8_t)dg[1][sl] << 8) |
                            ((uint32_t)(uint8_t)dg[2][sl] << 16) |
                            ((uint32_t)(uint8_t)dg[3][sl] << 24);
        *reinterpret_cast<uint32_t *>(d + sl * plane + r * kp + k0 + kk) = wv;
    }
}

}  // namespace

kfb_status oz_slice_colmajor(const double *src, long long rows, int K, long long ld,
                             const OzSlices &o, unsigned long long *scratch_max, cudaStream_t s) {
    KFB_TRY(oz_check(o, K));
    if (rows <= 0) return KFB_OK;
    KFB_TRY(zero(scratch_max, (size_t)rows * sizeof(unsigned long long), s));
    if (K > 0) {
        const int kchunk = 256;
        const dim3 gm((unsigned)((rows + 255) / 256), (unsigned)((K + kchunk - 1) / kchunk));
        colmajor_absmax_kernel<<<gm, 256, 0, s>>>(src, rows, K, ld, kchunk, scratch_max);
        KFB_CUDA_TRY(cudaGetLastError());
    }
    const dim3 gd((unsigned)((rows + 31) / 32), (unsigned)(o.kp / 32));
    switch (o.S) {
#define KFB_OZ_CM(SS)                                                                          \
    case SS:                                                                                   \
        colmajor_digits_kernel<SS><<<gd, 256, 0, s>>>(src, rows, K, ld, o.kp, scratch_max,    \
                                                      o.d, o.e);                               \
        break;
        KFB_OZ_CM(2)
        KFB_OZ_CM(3)
        KFB_OZ_CM(4)
        KFB_OZ_CM(5)
        KFB_OZ_CM(6)
        KFB_OZ_CM(7)
#undef KFB_OZ_CM
        default:
            return set_error(KFB_ERR_INVALID_ARG, "digit planes S=%d outside 2..%d", o.S, OZ_MAXS);
    }
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

int oz_gen_tiles(const OzGen &g, int S) {
    if (g.M <= 0 || g.N <= 0) return 0;
    const int BN = oz_bn(S);
    const int ntr = (g.M + BM - 1) / BM, ntc = (g.N + BN - 1) / BN;
    if (g.mode != OZ_GEN_LOWER) return ntr * ntc;
    int n = 0;
    for (int ti = 0; ti < ntr; ++ti) n += lower_tiles(ti, ntc, BN);
    return n;
}

namespace {
kfb_status oz_gemm_core(const OzSlices &A, const OzSlices &B, const OzTile *tiles,
                        const OzGen &gen, int ntiles, const OzEpi &epi, int *err,
                        cudaStream_t s) {
    if (ntiles <= 0) return KFB_OK;
    if (!device_is_sm100())
        return set_error(KFB_ERR_UNSUPPORTED, "the int8 tensor-core GEMM needs an sm_100 (B200) device");
    if (A.S != B.S || A.kp != B.kp)
        return set_error(KFB_ERR_INVALID_ARG, "digit planes of A and B differ (S %d/%d, kp %d/%d)",
                         A.S, B.S, A.kp, B.kp);
    KFB_TRY(oz_check(A, A.kp));
    if (A.S * A.rows >= (1LL << 31) || B.S * B.rows >= (1LL << 31))
        return set_error(KFB_ERR_INVALID_ARG, "digit planes too tall for a tensor map");
    DevBuf derr;
    int *e = err;
    if (!e) {
        KFB_TRY(derr.alloc(sizeof(int), s));
        KFB_TRY(zero(derr.ptr, sizeof(int), s));
        e = derr.as<int>();
    }
    switch (A.S) {
        case 2: KFB_TRY(launch<2>(A, B, tiles, gen, ntiles, epi, e, s)); break;
        case 3: KFB_TRY(launch<3>(A, B, tiles, gen, ntiles, epi, e, s)); break;
        case 4: KFB_TRY(launch<4>(A, B, tiles, gen, ntiles, epi, e, s)); break;
        case 5: KFB_TRY(launch<5>(A, B, tiles, gen, ntiles, epi, e, s)); break;
        case 6: KFB_TRY(launch<6>(A, B, tiles, gen, ntiles, epi, e, s)); break;
        case 7: KFB_TRY(launch<7>(A, B, tiles, gen, ntiles, epi, e, s)); break;
        default: return set_error(KFB_ERR_INVALID_ARG, "S=%d", A.S);
    }
    if (err) return KFB_OK;
    int herr = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&herr, e, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) return set_error(KFB_ERR_TIMEOUT, "int8 tensor-core GEMM: a pipeline wait timed out");
    return KFB_OK;
}
}  // namespace

kfb_status oz_gemm(const OzSlices &A, const OzSlices &B, const OzTile *tiles, int ntiles,
                   const OzEpi &epi, int *err, cudaStream_t s) {
    return oz_gemm_core(A, B, tiles, OzGen(), ntiles, epi, err, s);
}

kfb_status oz_gemm_gen(const OzSlices &A, const OzSlices &B, const OzGen &g, const OzEpi &epi,
                       int *err, cudaStream_t s) {
    return oz_gemm_core(A, B, nullptr, g, oz_gen_tiles(g, A.S), epi, err, s);
}

kfb_status oz_gemm_dense(const OzSlices &A, const OzSlices &B, int M, int N, const OzEpi &epi,
                         cudaStream_t s) {
    std::vector<OzTile> tiles;
    const int BN = oz_bn(A.S);
    for (int m0 = 0; m0 < M; m0 += BM)
        for (int n0 = 0; n0 < N; n0 += BN) {
            OzTile t{};
            t.a0 = m0;
            t.b0 = n0;
            t.m = std::min(BM, M - m0);
            t.n = std::min(BN, N - n0);
            t.c_off = (long long)m0 * epi.ldr + (long long)n0 * epi.ldc;
            tiles.push_back(t);
        }
    if (tiles.empty()) return KFB_OK;
    DevBuf dt;
    KFB_TRY(upload(dt, tiles, s));
    return oz_gemm(A, B, dt.as<OzTile>(), (int)tiles.size(), epi, nullptr, s);
}

}  // namespace kfb

// ---------------------------------------------------------------- C ABI
extern "C" kfb_status kfb_gemm_f64_i8(int m, int n, int k, double alpha, const double *a,
                                      int lda, const double *b, int ldb, double beta, double *c,
                                      int ldc, int slices, void *stream) {
    using namespace kfb;
    if (m < 0 || n < 0 || k < 0) return set_error(KFB_ERR_INVALID_ARG, "negative dimension");
    if (slices < 2 || slices > OZ_MAXS)
        return set_error(KFB_ERR_INVALID_ARG, "slices must be in 2..%d", OZ_MAXS);
    if (beta != 0.0 && beta != 1.0) return set_error(KFB_ERR_INVALID_ARG, "beta must be 0 or 1");
    if (k > 65536) return set_error(KFB_ERR_INVALID_ARG, "k must be <= 65536");
    if (m == 0 || n == 0) return KFB_OK;
    if (!a || !b || !c) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (lda < k || ldb < k || ldc < n) return set_error(KFB_ERR_INVALID_ARG, "leading dimension");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k == 0) {
        if (beta == 0.0) KFB_CUDA_TRY(cudaMemset2DAsync(c, (size_t)ldc * 8, 0, (size_t)n * 8, m, s));
        return KFB_OK;
    }
    OzSlices A, B;
    DevBuf da, db, dea, deb;
    A.S = B.S = slices;
    A.kp = B.kp = oz_kp(k);
    A.rows = m;
    B.rows = n;
    KFB_TRY(da.alloc((size_t)slices * m * A.kp, s));
    KFB_TRY(db.alloc((size_t)slices * n * B.kp, s));
    KFB_TRY(dea.alloc((size_t)m * sizeof(int), s));
    KFB_TRY(deb.alloc((size_t)n * sizeof(int), s));
    A.d = da.as<int8_t>();
    B.d = db.as<int8_t>();
    A.e = dea.as<int>();
    B.e = deb.as<int>();
    KFB_TRY(oz_slice_rows<double>(a, m, k, lda, A, s));
    KFB_TRY(oz_slice_rows<double>(b, n, k, ldb, B, s));
    OzEpi epi;
    epi.c = c;
    epi.ldr = ldc;
    epi.ldc = 1;
    epi.mode = beta == 0.0 ? OZ_STORE : OZ_ADD;
    epi.alpha = alpha;
    return oz_gemm_dense(A, B, m, n, epi, s);
}
