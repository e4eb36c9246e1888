// Allocation-free variant of the symmetric scalar kernel (FP64 CUDA cores).
//
// Some callers cannot allocate device memory during a call: a host framework
// that reserves the whole device-memory budget up front and hands the library
// only its inputs and outputs (a cudaMalloc inside the call would then fail),
// or a latency-critical loop that must not stall on the allocator, which
// cudaMalloc / cudaFree can do by synchronising the device.  For them,
// kfb_kernel_gaussian_symm_noalloc keeps all of its device scratch (packed
// same-label rows, their norms and molecule indices, the tile list) in one
// file-scope __device__ array of KFB_NOALLOC_SCRATCH_BYTES, which every GPU that
// loads the library holds until the process exits.  The caller still passes the
// descriptors and the output buffer.
//
// Set-up: the first call on a device looks up the device address of that array
// with cudaGetSymbolAddress (the host-side name of a __device__ array is only a
// stand-in and must never be passed to a kernel) while that device is current,
// and caches it per device.  Make that first call before any stream capture.
//
// All calls share the one array, which keeps the contents of the last call:
// every byte a call reads is written earlier in the same call (the output is
// zeroed with cudaMemsetAsync), and calls that overlap on the GPU -- on two
// streams, or from two host threads -- race on it.
#include <algorithm>
#include <cmath>
#include <mutex>

#include "kfb_internal.h"
#include "scalar_plan.h"
#include "scalar_simt_kernels.cuh"

namespace kfb {

namespace {

constexpr size_t NOALLOC_BYTES = (size_t)KFB_NOALLOC_SCRATCH_BYTES;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_setup_mutex;
void *g_scratch_ptr[MAX_DEVICES] = {};

// Device address of the scratch array for the current device.
kfb_status scratch_address(void **out) {
    int dev = 0;
    KFB_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES)
        return set_error(KFB_ERR_UNSUPPORTED, "device index %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p)
            return set_error(KFB_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
                             cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return KFB_OK;
}

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

template <class Tin>
kfb_status run(const ScalarProblem &p, const PairSink &sink, cudaStream_t s) {
    using T = double;
    std::vector<int> labels = collect_labels(p.s1, nullptr);
    Buckets bk = make_buckets(p.s1, labels);
    std::vector<PairTile> tiles = make_pair_tiles(bk, bk, true, simt::ST, simt::ST);
    const int R = bk.rows();
    const int Dp = (p.rep + simt::SK - 1) / simt::SK * simt::SK;
    // scratch layout: packed rows | norms | molecule index | source row | tiles
    const size_t off_norm = align256((size_t)R * Dp * sizeof(T));
    const size_t off_mol = off_norm + align256((size_t)R * sizeof(T));
    const size_t off_src = off_mol + align256((size_t)R * sizeof(int));
    const size_t off_tiles = off_src + align256((size_t)R * sizeof(int));
    const size_t need = off_tiles + align256(tiles.size() * sizeof(PairTile));
    if (need > NOALLOC_BYTES)
        return set_error(KFB_ERR_INVALID_ARG,
                         "kfb_kernel_gaussian_symm_noalloc: this problem needs %zu bytes of "
                         "scratch (%d packed atoms x %d); the fixed scratch array holds %zu bytes",
                         need, R, Dp, NOALLOC_BYTES);
    const size_t count = sink.layout == KFB_DENSE ? (size_t)sink.n * sink.n
                                                  : (size_t)sink.n * (sink.n + 1) / 2;
    KFB_CUDA_TRY(cudaMemsetAsync(sink.out, 0, count * sizeof(double), s));
    if (R == 0 || tiles.empty() || p.rep == 0) return KFB_OK;
    void *base = nullptr;
    KFB_TRY(scratch_address(&base));
    unsigned char *b = static_cast<unsigned char *>(base);
    T *packed = reinterpret_cast<T *>(b);
    T *norm = reinterpret_cast<T *>(b + off_norm);
    int *mol = reinterpret_cast<int *>(b + off_mol);
    int *src = reinterpret_cast<int *>(b + off_src);
    PairTile *dtiles = reinterpret_cast<PairTile *>(b + off_tiles);
    KFB_CUDA_TRY(cudaMemcpyAsync(mol, bk.mol.data(), R * sizeof(int), cudaMemcpyHostToDevice, s));
    KFB_CUDA_TRY(cudaMemcpyAsync(src, bk.src.data(), R * sizeof(int), cudaMemcpyHostToDevice, s));
    KFB_CUDA_TRY(cudaMemcpyAsync(dtiles, tiles.data(), tiles.size() * sizeof(PairTile),
                                 cudaMemcpyHostToDevice, s));
    const int rows_per_block = 8;
    simt::pack_rows_kernel<Tin, T><<<(R + rows_per_block - 1) / rows_per_block, 256, 0, s>>>(
        static_cast<const Tin *>(p.x1), src, R, p.rep, Dp, packed, norm);
    KFB_CUDA_TRY(cudaGetLastError());
    const T coef = T(-1.0 / (2.0 * p.sigma * p.sigma));
    simt::scalar_tile_kernel<T><<<(unsigned)tiles.size(), simt::SIMT_THREADS, 0, s>>>(
        packed, packed, Dp, norm, norm, mol, mol, dtiles, coef, sink);
    KFB_CUDA_TRY(cudaGetLastError());
    // the host vectors above are read by the copies before cudaMemcpyAsync
    // returns (pageable memory), so nothing here outlives the call
    return KFB_OK;
}

}  // namespace

}  // namespace kfb

using namespace kfb;

extern "C" kfb_status kfb_kernel_gaussian_symm_noalloc(const void *x, const int32_t *q,
                                                        const int32_t *n, int nm, int ma, int rep,
                                                        double sigma, kfb_dtype x_dt,
                                                        kfb_layout layout, void *out,
                                                        void *stream) {
    if (!std::isfinite(sigma) || sigma <= 0.0)
        return set_error(KFB_ERR_INVALID_ARG, "sigma must be > 0");
    if (layout != KFB_DENSE && layout != KFB_RFP_U && layout != KFB_RFP_L)
        return set_error(KFB_ERR_INVALID_ARG, "unknown layout %d", (int)layout);
    if (x_dt != KFB_F64 && x_dt != KFB_F32) return set_error(KFB_ERR_INVALID_ARG, "unknown dtype");
    if (nm < 0 || ma < 0 || rep < 0) return set_error(KFB_ERR_INVALID_ARG, "negative dimension");
    const size_t count = layout == KFB_DENSE ? (size_t)nm * nm : (size_t)nm * (nm + 1) / 2;
    if (count == 0) return KFB_OK;
    if (!x || !q || !n || !out) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    ScalarProblem p;
    p.x1 = p.x2 = x;
    p.s1 = p.s2 = SetView{q, n, nm, ma};
    p.rep = rep;
    p.sigma = sigma;
    p.x_dt = x_dt;
    p.symmetric = true;
    PairSink sink;
    sink.out = out;
    sink.out_f64 = 1;
    sink.mode = OUT_SYMM;
    sink.layout = layout;
    sink.n = nm;
    // run() sizes the problem against the scratch array before any device work
    if (x_dt == KFB_F64) return run<double>(p, sink, s);
    return run<float>(p, sink, s);
}
