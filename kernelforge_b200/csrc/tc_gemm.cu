// Grouped tcgen05 GEMM: C = A . B^T for a list of problems whose operands are
// row blocks / column windows of two K-major 2-D arrays, written through an
// ElemSink (dense, transposed or symmetric / RFP output).
//
// Operands are fp16 (or bf16) arrays; with NPROD = 3 each operand is a split
// pair x = hi + lo and the MMA issuer accumulates hi*hi + hi*lo + lo*hi (about
// 22 significant bits per operand, FP32 accumulation in TMEM).  Roles as in the
// scalar kernel: warp 0 TMA producer, warp 1 MMA issuer, warp 2 TMEM
// allocator, warps 4..11 epilogue (two per TMEM lane quadrant).  One persistent
// CTA per SM walks the tile list (problem, m0, n0).  All waits are bounded.
//
// Used for the Jacobian contraction (V . J^T per inner molecule) and the
// Hessian contraction (J_a^T . Y per molecule pair), which are the FLOP-heavy
// parts of src/local_kernels.cpp:791-974 and :1171-1900.
#include <cudaTypedefs.h>

#include <algorithm>
#include <climits>
#include <mutex>

#include "derivs.h"
#include "tc_common.cuh"
#include "tc_gemm.h"

namespace kfb {

namespace {

using namespace tc;

constexpr int BM = 128;
// Warps 0-3: TMA producer, MMA issuer, TMEM allocator, idle; then NEPI epilogue
// warps (NEPI / 4 column groups of four row quarters).  NEPI = 8 serves every
// epilogue mode with 64-element K blocks (128-byte swizzled rows); NEPI = 16
// only EPI_YSPLIT (short K, many stores): more warps in flight (register cap 96
// at 640 threads) and 32-element K blocks (64-byte swizzle), so that four
// stages fit next to its scratch.
constexpr int EPI_WARP0 = 4;

template <int NPROD, int NEPI, int BNT = 128>
struct Cfg {
    static constexpr int BN = BNT;  // tile columns (64: narrow-N problems, NEPI = 8 only)
    static constexpr int TMEM_COLS = 2 * BN;
    static constexpr int THREADS = 32 * (EPI_WARP0 + NEPI);
    static constexpr int BK = NEPI == 8 ? 64 : 32;
    static constexpr int TILE_A = BM * BK * 2, TILE_B = BN * BK * 2;
    static constexpr int STAGE_BUDGET = NEPI == 8 ? 196608 : 131072;
    static constexpr int NOP = NPROD == 3 ? 2 : 1;  // arrays per operand
    static constexpr int STAGE = NOP * (TILE_A + TILE_B);
    static constexpr int NSTAGE = STAGE_BUDGET / STAGE > 6 ? 6 : STAGE_BUDGET / STAGE;
    static constexpr int OFF_BARS = NSTAGE * STAGE;
    static constexpr int NBARS = 2 * NSTAGE + 5;
    static constexpr int OFF_TMEM = OFF_BARS + NBARS * 8;
    // NEPI = 16: the epilogue scratch is dynamic (static shared memory stops at
    // 48 KB), and launches of at most MAXP_SMEM problems read their problem
    // table (and tile starts) from a shared-memory copy
    // (rows of 36 floats: 16-byte aligned for the epilogue's vector reads)
    static constexpr int OFF_SCR = (OFF_TMEM + 16 + 15) / 16 * 16;
    static constexpr int SCR_LD = 36;
    static constexpr int MAXP_SMEM = NEPI == 8 ? 0 : 64;
    static constexpr int OFF_PROBS = OFF_SCR + (NEPI == 8 ? 0 : NEPI * 32 * SCR_LD * 4);
    static constexpr int OFF_TSTART = OFF_PROBS + MAXP_SMEM * (int)sizeof(TcProb);
    static constexpr int SMEM = OFF_TSTART + (MAXP_SMEM > 0 ? (MAXP_SMEM + 1) * 4 : 0) + 1024;
    static_assert(OFF_SCR % 16 == 0 && OFF_PROBS % 16 == 0, "shared-memory alignment");
    static_assert(SMEM <= 227 * 1024, "shared memory budget");
};

constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;

// K-major shared-memory descriptor of a BK-element (16-bit) row: 128-byte
// swizzle (8-row groups 1024 bytes apart) for BK = 64, 64-byte swizzle (512
// bytes apart) for BK = 32; sm_100 version bit.
template <int BK>
__device__ __forceinline__ uint64_t sdesc_k(uint32_t saddr) {
    if constexpr (BK == 64) {
        return sdesc(saddr);
    } else {
        static_assert(BK == 32, "K block");
        return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) |
               ((uint64_t)(512 >> 4) << 32) | ((uint64_t)1 << 46) | ((uint64_t)4 << 61);
    }
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 t = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&t);
}

__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity, int *err) {
    for (int i = 0; i < 64; ++i)
        if (mbar_try(bar, parity)) return true;
    const unsigned long long t0 = globaltimer();
    while (true) {
        if (mbar_try(bar, parity)) return true;
        if (*(volatile int *)err != 0) return false;
        if (globaltimer() - t0 > WAIT_LIMIT_NS) {
            atomicExch(err, 1);
            return false;
        }
    }
}

// Tile t of the launch: problems own consecutive tile ranges starting at
// tstart[p] (tstart[nprobs] = all tiles), row blocks outer, column blocks
// inner.  The largest p with tstart[p] <= t owns t (empty problems share their
// start with the next one and are skipped).
__device__ __forceinline__ TcTile tile_at(const TcProb *__restrict__ probs,
                                          const int *__restrict__ tstart, int nprobs, int t,
                                          int bn, bool n_outer = false) {
    int lo = 0, hi = nprobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (tstart[mid] <= t)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int loc = t - tstart[lo];
    if (n_outer) {
        const int ntm = (probs[lo].M + BM - 1) / BM;
        const int nt = loc / ntm;
        return TcTile{lo, (loc - nt * ntm) * BM, nt * bn, 0};
    }
    const int ntn = (probs[lo].N + bn - 1) / bn;
    const int mt = loc / ntn;
    return TcTile{lo, mt * BM, (loc - mt * ntn) * bn, 0};
}

template <int NPROD, int NEPI, int BNT>
__global__ void __launch_bounds__(Cfg<NPROD, NEPI, BNT>::THREADS, 1)
    tc_gemm_kernel(const __grid_constant__ CUtensorMap ta_hi, const __grid_constant__ CUtensorMap ta_lo,
                   const __grid_constant__ CUtensorMap tb_hi, const __grid_constant__ CUtensorMap tb_lo,
                   const TcProb *__restrict__ probs, const int *__restrict__ tstart, int nprobs, int ntiles,
                   uint32_t idesc, ElemSink sink, TcEpi epi, int *err) {
    using C = Cfg<NPROD, NEPI, BNT>;
    extern __shared__ uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t s_base = smem_u32(smem);
    const uint32_t bar0 = s_base + C::OFF_BARS;
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (C::NSTAGE + s); };
    auto tfull_bar = [&](int a) { return bar0 + 8u * (2 * C::NSTAGE + a); };
    auto tempty_bar = [&](int a) { return bar0 + 8u * (2 * C::NSTAGE + 2 + a); };
    const uint32_t done_bar = bar0 + 8u * (2 * C::NSTAGE + 4);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + C::OFF_TMEM);

    if (threadIdx.x == 0) {
        for (int s = 0; s < C::NSTAGE; ++s) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(tfull_bar(a), 1);
            mbar_init(tempty_bar(a), NEPI);
        }
        mbar_init(done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 2) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tmem_holder)),
                     "r"(C::TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    const TcProb *P = probs;
    const int *TS = tstart;
    if constexpr (C::MAXP_SMEM > 0) {
        if (nprobs <= C::MAXP_SMEM) {
            TcProb *ps = reinterpret_cast<TcProb *>(smem + C::OFF_PROBS);
            int *ts = reinterpret_cast<int *>(smem + C::OFF_TSTART);
            for (int i = threadIdx.x; i < nprobs; i += blockDim.x) ps[i] = probs[i];
            for (int i = threadIdx.x; i <= nprobs; i += blockDim.x) ts[i] = tstart[i];
            P = ps;
            TS = ts;
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = *tmem_holder;

    if (warp == 0) {
        if (lane == 0) {
            int stage = 0;
            uint32_t ph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const TcTile tl = tile_at(P, TS, nprobs, t, C::BN, NEPI == 16);
                const TcProb pb = P[tl.prob];
                const int nkb = (pb.K + C::BK - 1) / C::BK;
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!wait_bar(empty_bar(stage), ph ^ 1u, err)) {
                        ok = false;
                        break;
                    }
                    const uint32_t sa = s_base + stage * C::STAGE;
                    mbar_expect_tx(full_bar(stage), C::STAGE);
                    const int xa = pb.a_k0 + kb * C::BK, xb = pb.b_k0 + kb * C::BK;
                    tma_load_2d(sa, &ta_hi, xa, pb.a_row0 + tl.m0, full_bar(stage));
                    tma_load_2d(sa + C::NOP * C::TILE_A, &tb_hi, xb, pb.b_row0 + tl.n0,
                                full_bar(stage));
                    if (NPROD == 3) {
                        tma_load_2d(sa + C::TILE_A, &ta_lo, xa, pb.a_row0 + tl.m0,
                                    full_bar(stage));
                        tma_load_2d(sa + 2 * C::TILE_A + C::TILE_B, &tb_lo, xb, pb.b_row0 + tl.n0,
                                    full_bar(stage));
                    }
                    if (++stage == C::NSTAGE) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int stage = 0, acc = 0;
            uint32_t ph = 0, aph = 0;
            bool ok = true;
            for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
                const TcProb pb = P[tile_at(P, TS, nprobs, t, C::BN, NEPI == 16).prob];
                const int nkb = (pb.K + C::BK - 1) / C::BK;
                if (!wait_bar(tempty_bar(acc), aph ^ 1u, err)) break;
                tc_fence_after();
                const uint32_t dtm = tmem_base + (uint32_t)(acc * C::BN);
                for (int kb = 0; kb < nkb; ++kb) {
                    if (!wait_bar(full_bar(stage), ph, err)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = s_base + stage * C::STAGE;
                    const int nks = min(C::BK / 16, (pb.K - kb * C::BK) / 16);
                    for (int ks = 0; ks < nks; ++ks) {
                        const uint64_t ahi = sdesc_k<C::BK>(sa + ks * 32);
                        const uint64_t bhi = sdesc_k<C::BK>(sa + C::NOP * C::TILE_A + ks * 32);
                        umma_f16_idesc(dtm, ahi, bhi, idesc, (kb | ks) != 0 ? 1u : 0u);
                        if (NPROD == 3) {
                            const uint64_t alo = sdesc_k<C::BK>(sa + C::TILE_A + ks * 32);
                            const uint64_t blo =
                                sdesc_k<C::BK>(sa + 2 * C::TILE_A + C::TILE_B + ks * 32);
                            umma_f16_idesc(dtm, ahi, blo, idesc, 1u);
                            umma_f16_idesc(dtm, alo, bhi, idesc, 1u);
                        }
                    }
                    umma_commit(empty_bar(stage));
                    if (++stage == C::NSTAGE) {
                        stage = 0;
                        ph ^= 1u;
                    }
                }
                if (!ok) break;
                umma_commit(tfull_bar(acc));
                if (++acc == 2) {
                    acc = 0;
                    aph ^= 1u;
                }
            }
            umma_commit(done_bar);
            wait_bar(done_bar, 0, err);
        }
    } else if (warp >= EPI_WARP0) {
        const int q = warp & 3;
        const int h = (warp - EPI_WARP0) >> 2;  // column group
        constexpr int CPW = (C::BN / 32) / (NEPI / 4);  // 32-column chunks per warp
        __shared__ float molsum_static[NEPI == 8 ? NEPI : 1][32][33];
        float(*molsum_scr)[32][33] =
            NEPI == 8 ? molsum_static : reinterpret_cast<float(*)[32][33]>(smem + C::OFF_SCR);
        int acc = 0;
        uint32_t aph = 0;
        // the tile's problem (and for EPI_YSPLIT the (p, i) offset of this
        // lane's column); NEPI = 16 fetches them one tile ahead, so that the
        // dependent loads overlap the stores of the tile before
        TcTile tl_n{};
        TcProb pb_n{};
        long long cb_n = -1;
        auto fetch = [&](int t) {
            tl_n = tile_at(P, TS, nprobs, t, C::BN, NEPI == 16);
            pb_n = P[tl_n.prob];
            if constexpr (NEPI == 16) {
                const int nl = tl_n.n0 + h * 32 + lane;
                cb_n = -1;
                if (nl < pb_n.N) {
                    const int2 pi = epi.ymap[pb_n.b_row0 + nl];
                    if (pi.x >= 0)
                        cb_n = ((long long)pi.x * epi.y_ld2 * epi.y_ma1 + pi.y) * epi.y_rep;
                }
            }
        };
        if constexpr (NEPI == 16) {
            if ((int)blockIdx.x < ntiles) fetch(blockIdx.x);
        }
        for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
            if constexpr (NEPI == 8) fetch(t);
            const TcTile tl = tl_n;
            const TcProb pb = pb_n;
            const long long cb_t = cb_n;
            if constexpr (NEPI == 16) {
                if (t + (int)gridDim.x < ntiles) fetch(t + gridDim.x);
            }
            const bool got = wait_bar(tfull_bar(acc), aph, err);
            if (!__all_sync(0xffffffffu, got)) break;
            tc_fence_after();
            const int m = tl.m0 + q * 32 + lane;
            const bool mvalid = m < pb.M;
            const long long grow = (long long)pb.row_off + m;
            const uint32_t tbase = tmem_base + ((uint32_t)(q * 32) << 16) + (uint32_t)(acc * C::BN);
#pragma unroll 1
            for (int cc = 0; cc < CPW; ++cc) {
                const int c = h * CPW + cc;
                float v[32];
                tmem_ld32(tbase + (uint32_t)(c * 32), v);
                if constexpr (NEPI == 16) {  // one chunk per warp: release the accumulator now
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(tempty_bar(acc));
                }
                const int n0 = tl.n0 + c * 32;
                if (NEPI == 16 || epi.mode == EPI_YSPLIT) {
                    // lane l: the (p, i) part of column n0 + l's offset; the
                    // 32 x 32 block is turned in shared memory so that each lane
                    // writes 8 consecutive k of one column (octets never cross
                    // a c boundary: rep % 8 == 0) as 16 bytes of yhi and of ylo
                    long long cb = cb_t;
                    if constexpr (NEPI == 8) {
                        const int nl = n0 + lane;
                        cb = -1;
                        if (nl < pb.N) {
                            const int2 pi = epi.ymap[pb.b_row0 + nl];
                            if (pi.x >= 0)
                                cb = ((long long)pi.x * epi.y_ld2 * epi.y_ma1 + pi.y) * epi.y_rep;
                        }
                    }
                    // NEPI = 16: the block column-major in rows of 36 floats (the
                    // column j of 32 rows is row j of the scratch), so a lane's 8
                    // rows of one column are two 16-byte loads; the writes (bank
                    // 4 j + lane) and the loads (8 lanes of a phase: two columns,
                    // four octets) are free of bank conflicts
                    float *scrv = reinterpret_cast<float *>(smem + C::OFF_SCR) +
                                  (size_t)(warp - EPI_WARP0) * 32 * C::SCR_LD;
                    float(*scr)[33] = molsum_scr[warp - EPI_WARP0];
                    if constexpr (NEPI == 16) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) scrv[j * C::SCR_LD + lane] = v[j];
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) scr[lane][j] = v[j];
                    }
                    __syncwarp();
                    const int o = lane & 3;
                    const int mo = tl.m0 + q * 32 + o * 8;
                    const bool ovalid = mo < pb.M;
                    const int yc = mo / epi.y_rep;
                    const long long roff =
                        (long long)yc * epi.y_ma1 * epi.y_rep + (mo - yc * epi.y_rep);
                    const float alpha = (float)pb.alpha;
#pragma unroll
                    for (int g = 0; g < 4; ++g) {
                        const int j = g * 8 + (lane >> 2);
                        const long long base = __shfl_sync(0xffffffffu, cb, j);
                        if (!ovalid || base < 0) continue;
                        float xs[8];
                        if constexpr (NEPI == 16) {
                            const float4 x0 = *reinterpret_cast<const float4 *>(
                                scrv + j * C::SCR_LD + o * 8);
                            const float4 x1 = *reinterpret_cast<const float4 *>(
                                scrv + j * C::SCR_LD + o * 8 + 4);
                            xs[0] = x0.x; xs[1] = x0.y; xs[2] = x0.z; xs[3] = x0.w;
                            xs[4] = x1.x; xs[5] = x1.y; xs[6] = x1.z; xs[7] = x1.w;
                        } else {
#pragma unroll
                            for (int r = 0; r < 8; ++r) xs[r] = scr[o * 8 + r][j];
                        }
                        unsigned hw[4], lw[4];
#pragma unroll
                        for (int r = 0; r < 8; r += 2) {
                            const float2 x = make_float2(xs[r] * alpha, xs[r + 1] * alpha);
                            const __half2 hv = __float22half2_rn(x);
                            const float2 hf = __half22float2(hv);
                            const __half2 lv = __float22half2_rn(make_float2(x.x - hf.x, x.y - hf.y));
                            hw[r / 2] = *reinterpret_cast<const unsigned *>(&hv);
                            lw[r / 2] = *reinterpret_cast<const unsigned *>(&lv);
                        }
                        const size_t off = (size_t)(base + roff);
                        *reinterpret_cast<uint4 *>(epi.yhi + off) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                        *reinterpret_cast<uint4 *>(epi.ylo + off) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                    }
                    __syncwarp();  // scr is rewritten by the next chunk
                    continue;
                }
                if (epi.mode == EPI_SINK) {
                    if (mvalid) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const int n = n0 + j;
                            if (n < pb.N) {
                                if (epi.sink_t)
                                    sink_store(sink, pb.col_off + n, pb.row_off + m,
                                               (double)v[j] * pb.alpha, pb.diag);
                                else
                                    sink_store(sink, pb.row_off + m, pb.col_off + n,
                                               (double)v[j] * pb.alpha, pb.diag);
                            }
                        }
                    }
                    continue;
                }
                const int nvalid = min(32, pb.N - n0);
                const long long gcol0 = (long long)pb.col_off + n0;
                const float alpha = (float)pb.alpha;
                const bool vec = epi.vec && nvalid == 32;
                if (epi.mode == EPI_DENSE) {
                    if (nvalid <= 0) continue;  // warp-uniform
                    // bias: one coalesced load, then broadcast by shuffles
                    const float bl = (epi.bias && lane < nvalid) ? epi.bias[gcol0 + lane] : 0.f;
                    float z[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        z[j] = v[j] * alpha + __shfl_sync(0xffffffffu, bl, j);
                    float(*scr)[33] = molsum_scr[warp - EPI_WARP0];
                    const long long grow0 = (long long)pb.row_off + tl.m0 + q * 32;
                    const int mrows = min(32, pb.M - (tl.m0 + q * 32));  // valid rows of the chunk
                    if (epi.zf32 && epi.accumulate) {
                        if (mvalid) {
                            float *d = epi.zf32 + grow * epi.ld + gcol0;
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (j < nvalid) atomicAdd(d + j, z[j]);
                        }
                    } else if (epi.zf32) {
                        if (vec) {
                            // stage the 32 x 32 chunk, then 4 rows x 128 B per store
#pragma unroll
                            for (int j = 0; j < 32; ++j) scr[lane][j] = z[j];
                            __syncwarp();
                            const int rsub = lane >> 3, c4 = (lane & 7) * 4;
#pragma unroll
                            for (int rr = 0; rr < 8; ++rr) {
                                const int row = rr * 4 + rsub;
                                if (row < mrows)
                                    *reinterpret_cast<float4 *>(epi.zf32 + (grow0 + row) * epi.ld +
                                                                gcol0 + c4) =
                                        make_float4(scr[row][c4], scr[row][c4 + 1],
                                                    scr[row][c4 + 2], scr[row][c4 + 3]);
                            }
                            __syncwarp();
                        } else if (mvalid) {
                            float *d = epi.zf32 + grow * epi.ld + gcol0;
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (j < nvalid) d[j] = z[j];
                        }
                    }
                    if (epi.act || epi.act_t) {
#pragma unroll
                        for (int j = 0; j < 32; ++j) z[j] = cosf(z[j]);
                        if (epi.act) {
                            if (vec) {
                                // stage, then 8 rows x 64 B per store (16 B per lane)
#pragma unroll
                                for (int j = 0; j < 32; ++j) scr[lane][j] = z[j];
                                __syncwarp();
                                const int rsub = lane >> 2, c8 = (lane & 3) * 8;
#pragma unroll
                                for (int rr = 0; rr < 4; ++rr) {
                                    const int row = rr * 8 + rsub;
                                    if (row < mrows) {
                                        uint4 u;
                                        u.x = pack_bf16(scr[row][c8], scr[row][c8 + 1]);
                                        u.y = pack_bf16(scr[row][c8 + 2], scr[row][c8 + 3]);
                                        u.z = pack_bf16(scr[row][c8 + 4], scr[row][c8 + 5]);
                                        u.w = pack_bf16(scr[row][c8 + 6], scr[row][c8 + 7]);
                                        *reinterpret_cast<uint4 *>(epi.act + (grow0 + row) * epi.ld +
                                                                   gcol0 + c8) = u;
                                    }
                                }
                                __syncwarp();
                            } else if (mvalid) {
                                __nv_bfloat16 *d = epi.act + grow * epi.ld + gcol0;
#pragma unroll
                                for (int j = 0; j < 32; ++j)
                                    if (j < nvalid) d[j] = __float2bfloat16_rn(z[j]);
                            }
                        }
                        if (epi.act_t && mvalid) {
                            // lanes hold consecutive rows: these stores coalesce
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                if (j < nvalid)
                                    epi.act_t[(gcol0 + j) * epi.ld_t + grow] =
                                        __float2bfloat16_rn(z[j]);
                        }
                    }
                } else if (epi.mode == EPI_DSIN_T) {
                    if (nvalid <= 0 || !mvalid) continue;
                    const float *a = epi.aux + grow * epi.ld + gcol0;
                    float g[32];
                    if (vec) {
#pragma unroll
                        for (int j = 0; j < 32; j += 4) {
                            const float4 t4 = *reinterpret_cast<const float4 *>(a + j);
                            g[j] = t4.x;
                            g[j + 1] = t4.y;
                            g[j + 2] = t4.z;
                            g[j + 3] = t4.w;
                        }
                    } else {
#pragma unroll
                        for (int j = 0; j < 32; ++j) g[j] = j < nvalid ? a[j] : 0.f;
                    }
#pragma unroll
                    for (int j = 0; j < 32; ++j)
                        if (j < nvalid)
                            epi.act_t[(gcol0 + j) * epi.ld_t + grow] =
                                __float2bfloat16_rn(-v[j] * alpha * sinf(g[j]));
                } else {  // EPI_COS_MOLSUM, EPI_SIN_RUNSUM
                    // rows with one destination are consecutive: sum each run of rows
                    // per column through shared memory, one atomic add per (run, column)
                    float(*scr)[33] = molsum_scr[warp - EPI_WARP0];
                    const int mol = mvalid ? epi.mol[grow] : -1;
                    if (epi.mode == EPI_SIN_RUNSUM) {
                        // scale sin(aux[atom row, col]) times the product
                        const float *a =
                            epi.aux + (long long)(mvalid ? epi.atom[grow] : 0) * epi.ld_aux + gcol0;
                        float g[32];
                        if (vec) {
#pragma unroll
                            for (int j = 0; j < 32; j += 4) {
                                const float4 t4 = *reinterpret_cast<const float4 *>(a + j);
                                g[j] = t4.x;
                                g[j + 1] = t4.y;
                                g[j + 2] = t4.z;
                                g[j + 3] = t4.w;
                            }
                        } else {
#pragma unroll
                            for (int j = 0; j < 32; ++j) g[j] = (mvalid && j < nvalid) ? a[j] : 0.f;
                        }
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const bool ok = mvalid && j < nvalid;
                            scr[j][lane] = ok ? epi.scale * sinf(g[j]) * (v[j] * alpha) : 0.f;
                        }
                    } else {
                        const float bl = (epi.bias && lane < nvalid && nvalid > 0)
                                             ? epi.bias[gcol0 + lane]
                                             : 0.f;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const bool ok = mvalid && j < nvalid;
                            const float bias = __shfl_sync(0xffffffffu, bl, j);
                            scr[j][lane] = ok ? epi.scale * cosf(v[j] * alpha + bias) : 0.f;
                        }
                    }
                    __syncwarp();
                    // lane l owns column n0 + l and walks the 32 rows by molecule runs
                    const bool cok = lane < nvalid;
                    float *col = epi.molsum + gcol0 + lane;
                    float run = 0.f;
                    int cur = __shfl_sync(0xffffffffu, mol, 0);
                    for (int r = 0; r < 32; ++r) {
                        const int mr = __shfl_sync(0xffffffffu, mol, r);
                        if (mr != cur) {
                            if (cur >= 0 && cok) atomicAdd(col + (long long)cur * epi.ld, run);
                            run = 0.f;
                            cur = mr;
                        }
                        run += scr[lane][r];
                    }
                    if (cur >= 0 && cok) atomicAdd(col + (long long)cur * epi.ld, run);
                    __syncwarp();
                }
            }
            if constexpr (NEPI == 8) {
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(tempty_bar(acc));
            }
            if (++acc == 2) {
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
                     "r"(C::TMEM_COLS)
                     : "memory");
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encoder() {
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

kfb_status map2d(CUtensorMap *m, const void *ptr, long long rows, long long cols, int box_rows,
                 bool bf16, int box_cols = 64) {
    auto enc = encoder();
    if (!enc) return set_error(KFB_ERR_CUDA, "cuTensorMapEncodeTiled unavailable");
    if (cols % 8 != 0) return set_error(KFB_ERR_INVALID_ARG, "TMA operand rows must be 16-byte multiples");
    cuuint64_t gdim[2] = {(cuuint64_t)cols, (cuuint64_t)std::max<long long>(rows, 1)};
    cuuint64_t gstride[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, bf16 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT16,
                     2, const_cast<void *>(ptr), gdim, gstride, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE,
                     box_cols == 64 ? CU_TENSOR_MAP_SWIZZLE_128B : CU_TENSOR_MAP_SWIZZLE_64B,
                     CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(KFB_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return KFB_OK;
}

template <int NPROD, int NEPI, int BNT>
kfb_status launch_cfg(const CUtensorMap &ma_hi, const CUtensorMap &ma_lo, const CUtensorMap &mb_hi,
                      const CUtensorMap &mb_lo, const TcProb *probs, const int *tstart,
                      int nprobs, int ntiles, bool bf16, const ElemSink &sink, const TcEpi &e,
                      int *errp, cudaStream_t s) {
    using C = Cfg<NPROD, NEPI, BNT>;
    static bool done = false;
    if (!done) {
        KFB_CUDA_TRY(cudaFuncSetAttribute(tc_gemm_kernel<NPROD, NEPI, BNT>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, C::SMEM));
        done = true;
    }
    const int grid = std::min(ntiles, device_sm_count());
    const uint32_t idesc = make_idesc(BM, C::BN, bf16 ? 1 : 0);
    tc_gemm_kernel<NPROD, NEPI, BNT><<<grid, C::THREADS, C::SMEM, s>>>(
        ma_hi, ma_lo, mb_hi, mb_lo, probs, tstart, nprobs, ntiles, idesc, sink, e, errp);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

template <int NPROD>
kfb_status launch(const TcOperand &A, const TcOperand &B, bool bf16,
                  const std::vector<TcProb> &probs, const ElemSink &sink, const TcEpi &epi,
                  int *err_flag, cudaStream_t s) {
    const bool ysplit = epi.mode == EPI_YSPLIT;
    const bool narrow = !ysplit && epi.tile_n64;
    const int bn = narrow ? 64 : 128;
    std::vector<int> tstart(probs.size() + 1);
    long long ntiles = 0;
    for (int p = 0; p < (int)probs.size(); ++p) {
        const TcProb &pb = probs[p];
        if (pb.K % 16 != 0 || pb.a_k0 % 8 != 0 || pb.b_k0 % 8 != 0)
            return set_error(KFB_ERR_INVALID_ARG, "tc_gemm: K and column offsets must be multiples of 16 / 8");
        tstart[p] = (int)ntiles;
        if (pb.M > 0 && pb.N > 0)
            ntiles += (long long)((pb.M + BM - 1) / BM) * ((pb.N + bn - 1) / bn);
        if (ntiles >= INT_MAX) return set_error(KFB_ERR_INVALID_ARG, "tc_gemm: too many tiles");
    }
    tstart[probs.size()] = (int)ntiles;
    if (ntiles == 0) return KFB_OK;
    TcEpi e = epi;
    if (e.mode != EPI_SINK) {
        auto al = [](const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
        bool v = e.ld % 8 == 0 && al(e.zf32) && al(e.act) && al(e.aux);
        if (e.mode == EPI_SIN_RUNSUM) v = v && e.ld_aux % 4 == 0;
        for (const TcProb &pb : probs) v = v && pb.col_off % 8 == 0;
        e.vec = v ? 1 : 0;
    }
    const int bk = ysplit ? Cfg<NPROD, 16>::BK : Cfg<NPROD, 8>::BK;
    CUtensorMap ma_hi, ma_lo, mb_hi, mb_lo;
    KFB_TRY(map2d(&ma_hi, A.hi, A.rows, A.cols, BM, bf16, bk));
    KFB_TRY(map2d(&mb_hi, B.hi, B.rows, B.cols, bn, bf16, bk));
    if (NPROD == 3) {
        KFB_TRY(map2d(&ma_lo, A.lo, A.rows, A.cols, BM, bf16, bk));
        KFB_TRY(map2d(&mb_lo, B.lo, B.rows, B.cols, bn, bf16, bk));
    } else {
        ma_lo = ma_hi;
        mb_lo = mb_hi;
    }
    DevBuf dp, dt, derr;
    KFB_TRY(upload(dp, probs, s));
    KFB_TRY(upload(dt, tstart, s));
    int *errp = err_flag;
    if (!errp) {
        KFB_TRY(derr.alloc(sizeof(int), s));
        KFB_TRY(zero(derr.ptr, sizeof(int), s));
        errp = derr.as<int>();
    }
    if (ysplit)
        KFB_TRY((launch_cfg<NPROD, 16, 128>(ma_hi, ma_lo, mb_hi, mb_lo, dp.as<TcProb>(),
                                            dt.as<int>(), (int)probs.size(), (int)ntiles, bf16,
                                            sink, e, errp, s)));
    else if (narrow)
        KFB_TRY((launch_cfg<NPROD, 8, 64>(ma_hi, ma_lo, mb_hi, mb_lo, dp.as<TcProb>(),
                                          dt.as<int>(), (int)probs.size(), (int)ntiles, bf16,
                                          sink, e, errp, s)));
    else
        KFB_TRY((launch_cfg<NPROD, 8, 128>(ma_hi, ma_lo, mb_hi, mb_lo, dp.as<TcProb>(),
                                           dt.as<int>(), (int)probs.size(), (int)ntiles, bf16,
                                           sink, e, errp, s)));
    if (err_flag) return KFB_OK;
    int herr = 0;
    KFB_CUDA_TRY(cudaMemcpyAsync(&herr, derr.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    if (herr) return set_error(KFB_ERR_TIMEOUT, "tensor-core GEMM: a pipeline wait timed out");
    return KFB_OK;
}

// ---------------------------------------------------------------- packing
template <class T>
__global__ void absmax_kernel(const T *__restrict__ src, long long n, float *out) {
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        m = fmaxf(m, fabsf((float)src[i]));
    for (int o = 16; o; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    // non-negative floats order like their bit patterns
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(out), __float_as_int(m));
}

// max |dX[m][j][k][c]| over the real atoms of each molecule (j < nat[m],
// c < 3 nat[m]); padding entries are never read by the GEMMs and may hold
// anything
template <class T>
__global__ void absmax_dx_kernel(const T *__restrict__ dx, int ma, int rep,
                                 const int *__restrict__ nat, float *out) {
    const int m = blockIdx.y;
    const int na = min(max(nat[m], 0), ma);
    const int ld = 3 * ma, nc = 3 * na;
    const long long n = (long long)na * rep * nc;
    const T *base = dx + (size_t)m * ma * rep * ld;
    // warp per row (j, k), lanes over its 3 na columns
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const long long nrow = n / (nc > 0 ? nc : 1);
    float v = 0.f;
    for (long long row = (long long)blockIdx.x * nw + (threadIdx.x >> 5); row < nrow;
         row += (long long)gridDim.x * nw)
        for (int c = lane; c < nc; c += 32) v = fmaxf(v, fabsf((float)base[row * ld + c]));
    for (int o = 16; o; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(out), __float_as_int(v));
}

template <class T>
__global__ void split_rows_kernel(const T *__restrict__ src, long long n, float scale,
                                  __half *__restrict__ hi, __half *__restrict__ lo) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        const float v = (float)src[i] * scale;
        const __half h = __float2half_rn(v);
        hi[i] = h;
        lo[i] = __float2half_rn(v - __half2float(h));
    }
}

// Jt[(m, c)][(j, k)] = dX[m][j][k][c].  Tiles of 64 (j,k) x 32 c through
// shared memory (rows of dX read 128 bytes per warp, rows of Jt written as
// fp16 pairs, 128 bytes per warp); tiles wholly beyond the molecule's atoms
// (j >= nat[m] or c >= 3 nat[m]) are skipped: the GEMMs read (j, k) < nat rep
// only, and rows c >= 3 nat only feed output columns they discard.
constexpr int TDX_TILES = 8;

template <class T>
__global__ void __launch_bounds__(256) transpose_split_dx_kernel(
    const T *__restrict__ dx, int ma, int rep, const int *__restrict__ nat, float scale,
    __half *__restrict__ hi, __half *__restrict__ lo) {
    __shared__ float tile[64][33];
    const int m = blockIdx.z;
    const int ld = 3 * ma;
    const long long kk_total = (long long)ma * rep;
    const int c0 = blockIdx.y * 32;
    const int na = min(max(nat[m], 0), ma);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T *base = dx + (size_t)m * kk_total * ld;
    // TDX_TILES consecutive 64-row tiles per block (fewer, longer blocks)
    for (int tt = 0; tt < TDX_TILES; ++tt) {
        const long long kk0 = ((long long)blockIdx.x * TDX_TILES + tt) * 64;
        if (kk0 >= (long long)na * rep || c0 >= 3 * na) return;   // block-uniform
        if (tt > 0) __syncthreads();   // previous tile consumed
        for (int r = warp; r < 64; r += 8) {
            const long long kk = kk0 + r;
            const int c = c0 + lane;
            tile[r][lane] = (kk < kk_total && c < ld) ? (float)base[kk * ld + c] * scale : 0.f;
        }
        __syncthreads();
        const long long kk = kk0 + 2 * lane;
        for (int r = warp; r < 32; r += 8) {
            const int c = c0 + r;
            if (c >= ld) break;
            const size_t o = ((size_t)m * ld + c) * kk_total + kk;
            __half2 h, l;
            const float a0 = tile[2 * lane][r], a1 = tile[2 * lane + 1][r];
            h = __floats2half2_rn(a0, a1);
            const float2 back = __half22float2(h);
            l = __floats2half2_rn(a0 - back.x, a1 - back.y);
            if (kk + 1 < kk_total && (o & 1) == 0) {
                *reinterpret_cast<__half2 *>(hi + o) = h;
                *reinterpret_cast<__half2 *>(lo + o) = l;
            } else {
                if (kk < kk_total) {
                    hi[o] = __low2half(h);
                    lo[o] = __low2half(l);
                }
                if (kk + 1 < kk_total) {
                    hi[o + 1] = __high2half(h);
                    lo[o + 1] = __high2half(l);
                }
            }
        }
    }
}

// Jr[(m, j, c)][k] = dX[m][j][k][c] (one K-major row of rep per atom j and
// coordinate column c).  Tiles of 32 k x 32 c of one atom through shared
// memory; atoms j >= nat[m] and columns c >= 3 nat[m] are not written.
template <class T>
__global__ void __launch_bounds__(256) transpose_split_dx_rows_kernel(
    const T *__restrict__ dx, int ma, int rep, const int *__restrict__ nat,
    const int *__restrict__ blockmap, float scale, __half *__restrict__ hi,
    __half *__restrict__ lo) {
    __shared__ float tile[32][33];
    const int mj = blockIdx.x, m = mj / ma, j = mj - m * ma;
    const int na = min(max(nat[m], 0), ma);
    const int k0 = blockIdx.y * 32, c0 = blockIdx.z * 32;
    const int ld = 3 * ma;
    const int dst = blockmap ? blockmap[mj] : mj;  // block-uniform
    if (j >= na || c0 >= 3 * na || dst < 0) return;
    const T *base = dx + (size_t)mj * rep * ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < 32; r += 8) {
        const int k = k0 + r, c = c0 + lane;
        tile[r][lane] = (k < rep && c < ld) ? (float)base[(size_t)k * ld + c] * scale : 0.f;
    }
    __syncthreads();
    for (int r = warp; r < 32; r += 8) {
        const int c = c0 + r, k = k0 + lane;
        if (c >= ld || k >= rep) continue;
        const float v = tile[lane][r];
        const __half h = __float2half_rn(v);
        const size_t o = ((size_t)dst * ld + c) * rep + k;
        hi[o] = h;
        lo[o] = __float2half_rn(v - __half2float(h));
    }
}

// Yt[(p, c)][(i, k)] = Y[p][i][k][c], Y with row stride ld (the Hessian's
// per-pair Y blocks, ma1 x rep x ld each).
template <class T>
__global__ void transpose_split_y_kernel(const T *__restrict__ Y, int ma1, int rep, int ld,
                                         float scale, __half *__restrict__ hi,
                                         __half *__restrict__ lo) {
    __shared__ float tile[32][33];
    const int p = blockIdx.z;
    const long long kk_total = (long long)ma1 * rep;
    const long long kk0 = (long long)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    const T *base = Y + (size_t)p * kk_total * ld;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const long long kk = kk0 + r;
        const int c = c0 + threadIdx.x;
        tile[r][threadIdx.x] = (kk < kk_total && c < ld) ? (float)base[kk * ld + c] : 0.f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r;
        const long long kk = kk0 + threadIdx.x;
        if (c < ld && kk < kk_total) {
            const float v = tile[threadIdx.x][r] * scale;
            const __half h = __float2half_rn(v);
            const size_t o = ((size_t)p * ld + c) * kk_total + kk;
            hi[o] = h;
            lo[o] = __float2half_rn(v - __half2float(h));
        }
    }
}

}  // namespace

kfb_status tc_gemm_grouped(const TcOperand &A, const TcOperand &B, int nprod, bool bf16,
                           const std::vector<TcProb> &probs, const ElemSink &sink,
                           cudaStream_t s, const TcEpi &epi, int *err_flag) {
    if (!device_is_sm100())
        return set_error(KFB_ERR_UNSUPPORTED, "tensor-core GEMM needs an sm_100 (B200) device");
    if (nprod == 3) return launch<3>(A, B, bf16, probs, sink, epi, err_flag, s);
    return launch<1>(A, B, bf16, probs, sink, epi, err_flag, s);
}

// Power of two that brings the largest |value| to about 2^14: keeps the hi/lo
// fp16 pair out of fp16's subnormal range for the small entries (the pair
// then carries ~22 significant bits over ~28 binades below the maximum).
kfb_status pow2_from_device(const float *dmax, cudaStream_t s, float *scale) {
    float m = 0.f;
    KFB_CUDA_TRY(cudaMemcpyAsync(&m, dmax, sizeof(float), cudaMemcpyDeviceToHost, s));
    KFB_CUDA_TRY(cudaStreamSynchronize(s));
    *scale = 1.f;
    if (m > 0.f && std::isfinite(m)) *scale = std::ldexp(1.f, 14 - (int)std::ceil(std::log2(m)));
    return KFB_OK;
}

template <class T>
kfb_status pow2_scale(const T *src, long long n, cudaStream_t s, float *scale) {
    *scale = 1.f;
    if (n <= 0) return KFB_OK;
    DevBuf d;
    KFB_TRY(d.alloc(sizeof(float), s));
    KFB_TRY(zero(d.ptr, sizeof(float), s));
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 16);
    absmax_kernel<T><<<blocks, 256, 0, s>>>(src, n, d.as<float>());
    KFB_CUDA_TRY(cudaGetLastError());
    return pow2_from_device(d.as<float>(), s, scale);
}

template <class T>
kfb_status split_rows(const T *src, long long n, __half *hi, __half *lo, float *scale,
                      cudaStream_t s) {
    KFB_TRY(pow2_scale(src, n, s, scale));
    if (n <= 0) return KFB_OK;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 148LL * 64);
    split_rows_kernel<T><<<blocks, 256, 0, s>>>(src, n, *scale, hi, lo);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

template <class T>
kfb_status transpose_split_dx(const T *dx, int nm, int ma, int rep, const int *nat, __half *hi,
                              __half *lo, float *scale, cudaStream_t s) {
    const long long kk = (long long)ma * rep;
    *scale = 1.f;
    if (nm <= 0) return KFB_OK;
    {
        DevBuf d;
        KFB_TRY(d.alloc(sizeof(float), s));
        KFB_TRY(zero(d.ptr, sizeof(float), s));
        const long long per = kk * 3 * ma;
        const unsigned bx = (unsigned)std::min<long long>((per + 255) / 256, 64);
        absmax_dx_kernel<T><<<dim3(bx, (unsigned)nm), 256, 0, s>>>(dx, ma, rep, nat, d.as<float>());
        KFB_CUDA_TRY(cudaGetLastError());
        KFB_TRY(pow2_from_device(d.as<float>(), s, scale));
    }
    dim3 grid((unsigned)((kk + 64 * TDX_TILES - 1) / (64 * TDX_TILES)),
              (unsigned)((3 * ma + 31) / 32), (unsigned)nm);
    transpose_split_dx_kernel<T><<<grid, 256, 0, s>>>(dx, ma, rep, nat, *scale, hi, lo);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

template <class T>
kfb_status transpose_split_dx_rows(const T *dx, int nm, int ma, int rep, const int *nat,
                                   __half *hi, __half *lo, float *scale, cudaStream_t s,
                                   const int *blockmap) {
    *scale = 1.f;
    if (nm <= 0) return KFB_OK;
    {
        DevBuf d;
        KFB_TRY(d.alloc(sizeof(float), s));
        KFB_TRY(zero(d.ptr, sizeof(float), s));
        const long long per = (long long)ma * rep * 3 * ma;
        const unsigned bx = (unsigned)std::min<long long>((per + 255) / 256, 64);
        absmax_dx_kernel<T><<<dim3(bx, (unsigned)nm), 256, 0, s>>>(dx, ma, rep, nat, d.as<float>());
        KFB_CUDA_TRY(cudaGetLastError());
        KFB_TRY(pow2_from_device(d.as<float>(), s, scale));
    }
    dim3 grid((unsigned)(nm * ma), (unsigned)((rep + 31) / 32), (unsigned)((3 * ma + 31) / 32));
    transpose_split_dx_rows_kernel<T><<<grid, 256, 0, s>>>(dx, ma, rep, nat, blockmap, *scale,
                                                           hi, lo);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

template <class T>
kfb_status transpose_split_y(const T *Y, int np, int ma1, int rep, int ld, const float *amax,
                             __half *hi, __half *lo, float *scale, cudaStream_t s) {
    const long long kk = (long long)ma1 * rep;
    KFB_TRY(pow2_from_device(amax, s, scale));
    if (np <= 0) return KFB_OK;
    dim3 grid((unsigned)((kk + 31) / 32), (unsigned)((ld + 31) / 32), (unsigned)np);
    transpose_split_y_kernel<T><<<grid, dim3(32, 8), 0, s>>>(Y, ma1, rep, ld, *scale, hi, lo);
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

template kfb_status split_rows<float>(const float *, long long, __half *, __half *, float *,
                                      cudaStream_t);
template kfb_status split_rows<double>(const double *, long long, __half *, __half *, float *,
                                       cudaStream_t);
template kfb_status transpose_split_dx_rows<float>(const float *, int, int, int, const int *,
                                                   __half *, __half *, float *, cudaStream_t,
                                                   const int *);
template kfb_status transpose_split_dx<float>(const float *, int, int, int, const int *, __half *,
                                              __half *, float *, cudaStream_t);
template kfb_status transpose_split_dx<double>(const double *, int, int, int, const int *,
                                               __half *, __half *, float *, cudaStream_t);
template kfb_status transpose_split_y<float>(const float *, int, int, int, int, const float *,
                                             __half *, __half *, float *, cudaStream_t);
template kfb_status transpose_split_y<double>(const double *, int, int, int, int, const float *,
                                              __half *, __half *, float *, cudaStream_t);

}  // namespace kfb
