// Declarations of the derivative-kernel building blocks (derivs.cu).
#pragma once

#include "kernels_common.cuh"

namespace kfb {

// Element sink of the grouped GEMM: where C(R, C) of the global matrix goes.
enum ElemMode : int { EM_RECT = 0, EM_RECT_T = 1, EM_SYM = 2 };
constexpr int LAYOUT_DENSE_LOWER = 3;  // symmetric, lower triangle only

struct ElemSink {
    void *out = nullptr;
    int f64 = 1;
    int mode = EM_RECT;
    int layout = KFB_DENSE;  // EM_SYM: KFB_DENSE (both triangles), KFB_RFP_U/L, LAYOUT_DENSE_LOWER
    long long ld = 0;        // row stride (dense) or matrix order (RFP)
    int row_base = 0, col_base = 0;
};

struct GemmProb {
    const void *A;
    const void *B;
    long long lda, ldb;
    int M, N, K;
    int transA;
    int row_off, col_off;
    double alpha;
    int diag;
    int pad;
};

struct HessPair {
    int a, b, na, nb;
};

struct DerivSet {
    const void *x = nullptr;   // device (nm, ma, rep)
    const void *dx = nullptr;  // device (nm, ma, rep, 3 ma) or null
    SetView v;
};

__device__ __forceinline__ void sink_put(const ElemSink &s, long long idx, double v) {
    if (s.f64)
        static_cast<double *>(s.out)[idx] = v;
    else
        static_cast<float *>(s.out)[idx] = (float)v;
}

__device__ __forceinline__ void sink_store(const ElemSink &s, long long R, long long C, double v,
                                           int diag) {
    R += s.row_base;
    C += s.col_base;
    if (s.mode == EM_RECT) {
        sink_put(s, R * s.ld + C, v);
    } else if (s.mode == EM_RECT_T) {
        sink_put(s, C * s.ld + R, v);
    } else {
        if (diag && R > C) return;
        if (s.layout == KFB_DENSE) {
            sink_put(s, R * s.ld + C, v);
            if (R != C) sink_put(s, C * s.ld + R, v);
        } else if (s.layout == LAYOUT_DENSE_LOWER) {
            const long long hi = R > C ? R : C, lo = R > C ? C : R;
            sink_put(s, hi * s.ld + lo, v);
        } else {
            sink_put(s, sym_index((kfb_layout)s.layout, s.ld, R, C), v);
        }
    }
}

__device__ __forceinline__ void sink_add(const ElemSink &s, long long idx, double v) {
    if (s.f64)
        static_cast<double *>(s.out)[idx] += v;
    else
        static_cast<float *>(s.out)[idx] += (float)v;
}

// Calls f(idx) for every output index that sink_store(s, R, C, v, diag)
// writes (none, one, or the two mirrored entries of a dense symmetric sink).
template <class F>
__device__ __forceinline__ void sink_positions(const ElemSink &s, long long R, long long C,
                                               int diag, F f) {
    R += s.row_base;
    C += s.col_base;
    if (s.mode == EM_RECT) {
        f(R * s.ld + C);
    } else if (s.mode == EM_RECT_T) {
        f(C * s.ld + R);
    } else {
        if (diag && R > C) return;
        if (s.layout == KFB_DENSE) {
            f(R * s.ld + C);
            if (R != C) f(C * s.ld + R);
        } else if (s.layout == LAYOUT_DENSE_LOWER) {
            const long long hi = R > C ? R : C, lo = R > C ? C : R;
            f(hi * s.ld + lo);
        } else {
            f(sym_index((kfb_layout)s.layout, s.ld, R, C));
        }
    }
}

// tc: run the contraction GEMMs on the tensor cores (split fp16, three
// products); needs rep % 16 == 0 and an sm_100 device.
template <class T>
kfb_status jacobian_core(const DerivSet &outer, const DerivSet &inner, int rep, double sigma,
                         double alpha, bool tc, ElemSink sink, cudaStream_t s);

template <class T>
kfb_status hessian_core(const DerivSet &s1, const DerivSet &s2, int rep, double sigma,
                        bool symmetric, bool tc, ElemSink sink, cudaStream_t s);

}  // namespace kfb
