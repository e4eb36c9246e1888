// Device helpers shared by the scalar and derivative kernels.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kfb_internal.h"

namespace kfb {

// Tile of two label buckets: packed rows [a0, a_end) x [b0, b_end), at most
// the kernel's tile height each; `diag` marks a diagonal tile of a symmetric
// problem (both operands the same rows).
struct PairTile {
    int a0, a_end, b0, b_end, diag, pad0, pad1, pad2;
};

__device__ __forceinline__ void atomic_add_out(const PairSink &s, long long idx, double v) {
    if (s.out_f64)
        atomicAdd(static_cast<double *>(s.out) + idx, v);
    else
        atomicAdd(static_cast<float *>(s.out) + idx, (float)v);
}

// Commit the sum over one (molecule a) x (molecule b) rectangle of atom pairs.
// Symmetric problems keep the pairs with a <= b: a diagonal tile holds both
// (i, j) and (j, i), so pairs with a > b are dropped there; an off-diagonal
// tile holds (i, j) only, so a == b sums are doubled (the reference's
// "self-kernel cross-block pairs counted twice", src/local_kernels.cpp:565-566).
__device__ __forceinline__ void emit_pair(const PairSink &s, int a, int b, double v, int diag) {
    v *= s.scale;
    if (s.mode == OUT_RECT) {
        atomic_add_out(s, (long long)(a + s.row_off) * s.n + (b + s.col_off), v);
        return;
    }
    if (diag) {
        if (a > b) return;
    } else if (a == b) {
        v *= 2.0;
    }
    const long long r = a + s.row_off, c = b + s.col_off;
    if (s.layout == KFB_DENSE) {
        atomic_add_out(s, r * s.n + c, v);
        if (r != c) atomic_add_out(s, c * s.n + r, v);
    } else {
        atomic_add_out(s, sym_index((kfb_layout)s.layout, s.n, r, c), v);
    }
}

template <class T> __device__ __forceinline__ T kexp(T x);
template <> __device__ __forceinline__ double kexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float kexp<float>(float x) { return __expf(x); }

}  // namespace kfb
