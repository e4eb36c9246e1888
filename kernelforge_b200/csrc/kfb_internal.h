// Internal declarations shared by the libkfb translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "kfb.h"

namespace kfb {

// ---------------------------------------------------------------------------
// Errors: every entry point returns a kfb_status and records a message.
// ---------------------------------------------------------------------------
kfb_status set_error(kfb_status st, const char *fmt, ...);
const char *last_error();

#define KFB_CUDA_TRY(expr)                                                                  \
    do {                                                                                    \
        cudaError_t _e = (expr);                                                            \
        if (_e != cudaSuccess)                                                              \
            return ::kfb::set_error(KFB_ERR_CUDA, "%s failed: %s (%s:%d)", #expr,           \
                                    cudaGetErrorString(_e), __FILE__, __LINE__);            \
    } while (0)

#define KFB_TRY(expr)                                                                       \
    do {                                                                                    \
        kfb_status _s = (expr);                                                             \
        if (_s != KFB_OK) return _s;                                                        \
    } while (0)

// ---------------------------------------------------------------------------
// Stream-ordered scratch buffer (cudaMallocAsync / cudaFreeAsync).
// ---------------------------------------------------------------------------
struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    kfb_status alloc(size_t nbytes, cudaStream_t s);
    void release();
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Copy a host vector to a fresh device buffer on `s` (the host vector must stay
// alive until the stream reaches the copy; callers keep it in scope and the
// copy is issued from pageable memory, which the runtime stages synchronously).
template <class T>
kfb_status upload(DevBuf &buf, const std::vector<T> &v, cudaStream_t s) {
    KFB_TRY(buf.alloc(v.size() * sizeof(T) + 16, s));
    if (!v.empty())
        KFB_CUDA_TRY(cudaMemcpyAsync(buf.ptr, v.data(), v.size() * sizeof(T),
                                     cudaMemcpyHostToDevice, s));
    return KFB_OK;
}

// ---------------------------------------------------------------------------
// Host-side plan: atoms bucketed by label, molecules kept in order inside a
// bucket (the device analogue of the reference's PackedLabel /
// PackedLabelSym, src/local_kernels.cpp:61-149, :325-375).
// ---------------------------------------------------------------------------
struct SetView {
    const int32_t *q = nullptr;  // host (nm, ma)
    const int32_t *n = nullptr;  // host (nm,)
    int nm = 0, ma = 0;
    int natoms(int m) const {
        int v = n[m];
        return v < 0 ? 0 : (v > ma ? ma : v);
    }
};

struct Buckets {
    std::vector<int> labels;     // distinct labels, ascending
    std::vector<int> lab_start;  // packed row range of label l: [lab_start[l], lab_start[l+1])
    std::vector<int> src;        // packed row -> padded row index (m * ma + atom)
    std::vector<int> mol;        // packed row -> molecule index
    int rows() const { return (int)src.size(); }
};

// Distinct labels present in the active atoms of one or two sets
// (collect_distinct_labels_T, src/local_kernels.cpp:31-58).
std::vector<int> collect_labels(const SetView &a, const SetView *b);
// Bucket one set by the given label list.
Buckets make_buckets(const SetView &s, const std::vector<int> &labels);
// Derivative-axis offsets: offs[m] = 3 * sum_{m' < m} n[m'], returns naq.
long long deriv_offsets(const SetView &s, std::vector<int> &offs);

// ---------------------------------------------------------------------------
// RFP index maps (TRANSR='N'); usable on host and device.
// ---------------------------------------------------------------------------
// Fortran UPLO='U', i <= j (src/local_kernels.cpp:386-400).
__host__ __device__ inline long long rfp_upper(long long n, long long i, long long j) {
    const long long k = n / 2;
    const long long stride = (n & 1) ? n : n + 1;
    return (j >= k) ? (j - k) * stride + i : i * stride + (j + k + 1);
}
// Fortran UPLO='L', i >= j (src/cuda_local_kernels.cu:3148-3162).
__host__ __device__ inline long long rfp_lower(long long n, long long i, long long j) {
    if (n & 1) {
        const long long n1 = (n + 1) / 2;
        return (j < n1) ? i + j * n : n + (j - n1) + (i - n1) * n;
    }
    const long long nk = n / 2;
    return (j < nk) ? 1 + i + j * (n + 1) : (j - nk) + (i - nk) * (n + 1);
}
// Position of the symmetric element (r, c) in the requested layout.
__host__ __device__ inline long long sym_index(kfb_layout layout, long long n, long long r,
                                                long long c) {
    const long long lo = r < c ? r : c, hi = r < c ? c : r;
    if (layout == KFB_RFP_U) return rfp_upper(n, lo, hi);
    if (layout == KFB_RFP_L) return rfp_lower(n, hi, lo);
    return r * n + c;
}

// ---------------------------------------------------------------------------
// Output sink for molecule-pair sums (see kernels_common.cuh).
// ---------------------------------------------------------------------------
enum OutMode : int {
    OUT_RECT = 0,   // K[a * ld + b] (asymmetric sets)
    OUT_SYMM = 1    // symmetric: a <= b reduction rules, layout below
};

struct PairSink {
    void *out = nullptr;
    int out_f64 = 0;       // 1: double output, 0: float
    int mode = OUT_RECT;
    int layout = KFB_DENSE;
    long long n = 0;       // matrix order (symmetric) or row stride (rect)
    int row_off = 0;       // offset added to the molecule indices (full kernels)
    int col_off = 0;
    double scale = 1.0;    // multiplies every contribution
};

// ---------------------------------------------------------------------------
// Scalar-kernel launchers (scalar_simt.cu / scalar_tc.cu).
// ---------------------------------------------------------------------------
struct ScalarProblem {
    const void *x1 = nullptr, *x2 = nullptr;  // device, padded
    SetView s1, s2;
    int rep = 0;
    double sigma = 1.0;
    kfb_dtype x_dt = KFB_F64;
    bool symmetric = false;
};

kfb_status scalar_simt(const ScalarProblem &p, kfb_precision prec, const PairSink &sink,
                       cudaStream_t stream);
kfb_status scalar_tc(const ScalarProblem &p, const PairSink &sink, cudaStream_t stream);
// Symmetric split-fp16 kernel with X in host memory: chunked copies overlapped
// with the tile waves whose rows have arrived (scalar_tc.cu).
kfb_status scalar_tc_from_host(const ScalarProblem &p, const void *x_host, const PairSink &sink,
                               cudaStream_t stream);

// Zero an output region.
kfb_status zero(void *ptr, size_t bytes, cudaStream_t s);

int device_sm_count();
bool device_is_sm100();

// Optional event timing of the main tile kernel of a call (kfb_set_timing).
bool timing_enabled();
struct KernelTimer {
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaStream_t stream = nullptr;
    explicit KernelTimer(cudaStream_t s);
    ~KernelTimer();
    void start();
    void stop();
};

// Host-phase tracing (environment KFB_TRACE): 1 prints the host wall time of
// each traced phase to stderr; 2 also synchronises the stream at both ends of
// the phase, so the time includes the device work the phase enqueued.
int trace_level();
// Code-path log of this thread (kfb_path_log_*): the name of each path a call
// chose where it picks one of several (capped at a few KB).
void note_path(const char *name);
struct TraceScope {
    const char *name;
    cudaStream_t stream;
    double t0 = 0.0;
    int level = 0;
    TraceScope(const char *n, cudaStream_t s);
    ~TraceScope();
};

}  // namespace kfb
