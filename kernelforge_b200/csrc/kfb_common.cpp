// Host-side helpers of libkfb: error reporting, scratch buffers, label
// bucketing and derivative offsets.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <set>

#include "kfb_internal.h"

namespace kfb {

static thread_local std::string g_last_error;

kfb_status set_error(kfb_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

const char *last_error() { return g_last_error.c_str(); }

// The device's default memory pool returns unused memory to the driver at every
// synchronisation unless told otherwise; the solves synchronise between
// iterations, so their scratch (hundreds of MB) would be unmapped and mapped
// again on every call, and the derivative kernels' chunk buffers (tens of GB on
// a 180 GB device) would be remapped per call.  Keep up to KFB_POOL_KEEP_GB
// (default 64) GB in the pool.
static void keep_pool_memory() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return;
    std::lock_guard<std::mutex> lk(mu);
    if (done[dev]) return;
    done[dev] = true;
    const char *v = std::getenv("KFB_POOL_KEEP_GB");
    const double gb = v ? std::atof(v) : 64.0;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) != cudaSuccess) {
        (void)cudaGetLastError();
        return;
    }
    unsigned long long keep = (unsigned long long)((gb > 0 ? gb : 0.0) * (double)(1ull << 30));
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep) != cudaSuccess)
        (void)cudaGetLastError();
}

kfb_status DevBuf::alloc(size_t nbytes, cudaStream_t s) {
    release();
    keep_pool_memory();
    stream = s;
    bytes = nbytes ? nbytes : 16;
    cudaError_t e = cudaMallocAsync(&ptr, bytes, s);
    if (e != cudaSuccess) {
        ptr = nullptr;
        (void)cudaGetLastError();
        return set_error(KFB_ERR_ALLOC, "cudaMallocAsync(%zu bytes) failed: %s", bytes,
                         cudaGetErrorString(e));
    }
    return KFB_OK;
}

void DevBuf::release() {
    if (ptr) cudaFreeAsync(ptr, stream);
    ptr = nullptr;
    bytes = 0;
}

// Labels are nuclear charges or element indices: small non-negative integers
// take a direct table, anything else a sorted set.
static constexpr int LABEL_TABLE = 4096;

std::vector<int> collect_labels(const SetView &a, const SetView *b) {
    std::vector<unsigned char> seen(LABEL_TABLE, 0);
    std::set<int> other;
    auto scan = [&](const SetView &v) {
        for (int m = 0; m < v.nm; ++m) {
            const int32_t *q = v.q + (size_t)m * v.ma;
            const int na = v.natoms(m);
            for (int i = 0; i < na; ++i) {
                const int l = q[i];
                if (l >= 0 && l < LABEL_TABLE) seen[l] = 1;
                else other.insert(l);
            }
        }
    };
    scan(a);
    if (b) scan(*b);
    std::vector<int> out;
    for (int l : other)
        if (l < 0) out.push_back(l);
    for (int l = 0; l < LABEL_TABLE; ++l)
        if (seen[l]) out.push_back(l);
    for (int l : other)
        if (l >= LABEL_TABLE) out.push_back(l);
    return out;  // ascending
}

Buckets make_buckets(const SetView &s, const std::vector<int> &labels) {
    Buckets bk;
    bk.labels = labels;
    const int L = (int)labels.size();
    std::vector<int> table(LABEL_TABLE, -1);
    for (int l = 0; l < L; ++l)
        if (labels[l] >= 0 && labels[l] < LABEL_TABLE) table[labels[l]] = l;
    auto lidx = [&](int lbl) -> int {
        if (lbl >= 0 && lbl < LABEL_TABLE) return table[lbl];
        const auto it = std::lower_bound(labels.begin(), labels.end(), lbl);
        return (it != labels.end() && *it == lbl) ? (int)(it - labels.begin()) : -1;
    };
    // label of each active atom, counted in one pass
    std::vector<int> count(L + 1, 0);
    for (int m = 0; m < s.nm; ++m) {
        const int32_t *q = s.q + (size_t)m * s.ma;
        const int na = s.natoms(m);
        for (int i = 0; i < na; ++i) {
            const int l = lidx(q[i]);
            if (l >= 0) count[l + 1]++;
        }
    }
    bk.lab_start.assign(L + 1, 0);
    for (int l = 0; l < L; ++l) bk.lab_start[l + 1] = bk.lab_start[l] + count[l + 1];
    const int R = bk.lab_start[L];
    bk.src.resize(R);
    bk.mol.resize(R);
    std::vector<int> fill(bk.lab_start.begin(), bk.lab_start.end() - 1);
    for (int m = 0; m < s.nm; ++m) {
        const int32_t *q = s.q + (size_t)m * s.ma;
        const int na = s.natoms(m);
        for (int i = 0; i < na; ++i) {
            const int l = lidx(q[i]);
            if (l < 0) continue;
            const int r = fill[l]++;
            bk.src[r] = m * s.ma + i;
            bk.mol[r] = m;
        }
    }
    return bk;
}

long long deriv_offsets(const SetView &s, std::vector<int> &offs) {
    offs.resize(s.nm + 1);
    long long acc = 0;
    for (int m = 0; m < s.nm; ++m) {
        offs[m] = (int)acc;
        acc += 3LL * s.natoms(m);
    }
    offs[s.nm] = (int)acc;
    return acc;
}

kfb_status zero(void *ptr, size_t bytes, cudaStream_t s) {
    if (bytes) KFB_CUDA_TRY(cudaMemsetAsync(ptr, 0, bytes, s));
    return KFB_OK;
}

int device_sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

static bool g_timing = false;
static thread_local double g_last_ms = 0.0;

bool timing_enabled() { return g_timing; }

KernelTimer::KernelTimer(cudaStream_t s) : stream(s) {
    if (!g_timing) return;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
}
KernelTimer::~KernelTimer() {
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
}
void KernelTimer::start() {
    if (t0) cudaEventRecord(t0, stream);
}
void KernelTimer::stop() {
    if (!t1) return;
    cudaEventRecord(t1, stream);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    g_last_ms = ms;
}

double last_kernel_ms() { return g_last_ms; }
void set_timing(bool on) { g_timing = on; }

bool device_is_sm100() {
    int dev = 0, major = 0, minor = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, dev);
    return major == 10 && minor == 0;
}

int trace_level() {
    static const int lvl = [] {
        const char *v = std::getenv("KFB_TRACE");
        return v ? std::atoi(v) : 0;
    }();
    return lvl;
}

static thread_local std::string g_path_log;

void note_path(const char *name) {
    if (g_path_log.size() > 4096) return;
    if (!g_path_log.empty()) g_path_log += ',';
    g_path_log += name;
}

void path_log_clear() { g_path_log.clear(); }
const std::string &path_log() { return g_path_log; }

static double now_ms() {
    using namespace std::chrono;
    return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

TraceScope::TraceScope(const char *n, cudaStream_t s) : name(n), stream(s), level(trace_level()) {
    if (level <= 0) return;
    if (level >= 2) cudaStreamSynchronize(stream);
    t0 = now_ms();
}

TraceScope::~TraceScope() {
    if (level <= 0) return;
    if (level >= 2) cudaStreamSynchronize(stream);
    std::fprintf(stderr, "[kfb-trace] %-28s %9.3f ms\n", name, now_ms() - t0);
}

}  // namespace kfb
