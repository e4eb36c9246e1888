// Device code of the CUDA-core (FP64 / FP32) scalar tile kernel, shared by the
// launchers in scalar_simt.cu and scalar_noalloc.cu.
#pragma once

#include "kernels_common.cuh"

namespace kfb {
namespace simt {

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

// 128 threads: thread (ty = tid / 16, tx = tid % 16) owns rows 8 ty .. 8 ty + 7
// and columns 4 tx .. 4 tx + 3 of the 64 x 64 tile (12 shared loads per 32
// FMAs in the K loop).
constexpr int SIMT_THREADS = 128;

template <class T>
__global__ void __launch_bounds__(SIMT_THREADS) scalar_tile_kernel(
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
    const int tx = tid & 15, ty = tid >> 4;   // ty < 8
    const int nra = min(ST, t.a_end - t.a0);
    const int nrb = min(ST, t.b_end - t.b0);

    T acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = T(0);

    const int lr = tid >> 1, lk = (tid & 1) * 8;  // loader: row, first k
    for (int k0 = 0; k0 < Dp; k0 += SK) {
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int k = k0 + lk + u;
            As[lk + u][lr] = (lr < nra && k < Dp) ? A[(size_t)(t.a0 + lr) * Dp + k] : T(0);
            Bs[lk + u][lr] = (lr < nrb && k < Dp) ? B[(size_t)(t.b0 + lr) * Dp + k] : T(0);
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < SK; ++kk) {
            T a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = As[kk][ty * 8 + i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx * 4 + j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }

    // e_ij into shared memory (zero outside the valid rows / columns)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int r = ty * 8 + i;
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

}  // namespace simt
}  // namespace kfb
