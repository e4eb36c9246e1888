// extern "C" entry points of libkfb (declared in include/kfb.h): argument
// validation in the reference's terms, output zeroing, and dispatch to the
// scalar, derivative and solver launchers.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "derivs.h"
#include "kfb_internal.h"

namespace kfb {
kfb_status rfp_add_diag(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt, cudaStream_t s);
kfb_status full_to_rfp(const void *A, int n, kfb_layout uplo, kfb_dtype dt, void *arf, cudaStream_t s);
kfb_status rfp_to_full(const void *arf, int n, kfb_layout uplo, kfb_dtype dt, void *A, cudaStream_t s);
kfb_status rfp_potrf(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt, int *info, cudaStream_t s);
kfb_status rfp_potrs(const void *arf, void *B, int n, int nrhs, kfb_layout uplo, kfb_dtype dt, cudaStream_t s);
kfb_status cho_solve_rfp_f64(double *arf, const double *y, int n, double l2, kfb_layout uplo,
                             double *alpha, int *info, cudaStream_t s);
kfb_status feature_gramian(const float *z, const double *y, int nm, int d, kfb_layout layout,
                           float *ztz, double *zty, cudaStream_t s);
kfb_status ridge_solve_mixed(const float *zf, const double *y, int nm, int d, double l2,
                             double tol, int maxit, int flags, double *w, kfb_solve_info *info,
                             cudaStream_t s);
kfb_status krr_solve_mixed(const float *k_rfp, const double *y, int n, double l2, kfb_layout uplo,
                           double tol, int maxit, int flags, double *alpha, kfb_solve_info *info,
                           cudaStream_t s);
double last_kernel_ms();
void set_timing(bool on);
void path_log_clear();
const std::string &path_log();
}  // namespace kfb

using namespace kfb;

namespace {

inline cudaStream_t as_stream(void *s) { return static_cast<cudaStream_t>(s); }
inline size_t esize(kfb_dtype dt) { return dt == KFB_F64 ? 8 : 4; }

kfb_status check_sigma(double sigma) {
    if (!std::isfinite(sigma) || sigma <= 0.0)
        return set_error(KFB_ERR_INVALID_ARG, "sigma must be > 0");
    return KFB_OK;
}

kfb_status check_set(const void *x, const int32_t *q, const int32_t *n, int nm, int ma,
                     const char *name) {
    if (nm < 0 || ma < 0) return set_error(KFB_ERR_INVALID_ARG, "%s: negative dimension", name);
    if (nm > 0 && ma > 0 && (!x || !q || !n))
        return set_error(KFB_ERR_INVALID_ARG, "%s: null pointer", name);
    return KFB_OK;
}

kfb_status check_layout(kfb_layout l) {
    if (l != KFB_DENSE && l != KFB_RFP_U && l != KFB_RFP_L)
        return set_error(KFB_ERR_INVALID_ARG, "unknown layout %d", (int)l);
    return KFB_OK;
}

kfb_status check_prec(kfb_precision p) {
    if (p != KFB_PREC_FP64 && p != KFB_PREC_FP32 && p != KFB_PREC_SPLIT_F16)
        return set_error(KFB_ERR_INVALID_ARG, "unknown precision %d", (int)p);
    return KFB_OK;
}

SetView view(const int32_t *q, const int32_t *n, int nm, int ma) {
    SetView v;
    v.q = q;
    v.n = n;
    v.nm = nm;
    v.ma = ma;
    return v;
}

kfb_status scalar_dispatch(const ScalarProblem &p, kfb_precision prec, const PairSink &sink,
                           cudaStream_t s) {
    if (p.rep <= 0) return KFB_OK;
    if (prec == KFB_PREC_SPLIT_F16) return scalar_tc(p, sink, s);
    return scalar_simt(p, prec, sink, s);
}

// Derivative kernels compute in the element type of their inputs; the
// precision argument only selects the scalar block's arithmetic.
kfb_status check_deriv_prec(kfb_dtype dt, kfb_precision prec) {
    KFB_TRY(check_prec(prec));
    if (dt != KFB_F64 && dt != KFB_F32) return set_error(KFB_ERR_INVALID_ARG, "unknown dtype");
    return KFB_OK;
}

kfb_status naq_check(const SetView &v, long long naq, const char *message) {
    std::vector<int> offs;
    if (deriv_offsets(v, offs) != naq) return set_error(KFB_ERR_INVALID_ARG, "%s", message);
    return KFB_OK;
}

// The split-fp16 precision runs the derivative kernels' contraction GEMMs on the
// tensor cores when rep is a multiple of 16 (TMA rows of whole 16-byte units);
// otherwise, and for the FP64 / FP32 precisions, they run on CUDA cores.
bool use_tc(kfb_precision prec, int rep) {
    return prec == KFB_PREC_SPLIT_F16 && rep % 16 == 0 && device_is_sm100();
}

kfb_status jac_any(kfb_dtype dt, kfb_precision prec, const DerivSet &outer,
                   const DerivSet &inner, int rep, double sigma, double alpha,
                   const ElemSink &sink, cudaStream_t s) {
    if (rep <= 0) return KFB_OK;
    const bool tc = use_tc(prec, rep);
    if (dt == KFB_F64) return jacobian_core<double>(outer, inner, rep, sigma, alpha, tc, sink, s);
    return jacobian_core<float>(outer, inner, rep, sigma, alpha, tc, sink, s);
}

kfb_status hess_any(kfb_dtype dt, kfb_precision prec, const DerivSet &s1, const DerivSet &s2,
                    int rep, double sigma, bool symmetric, const ElemSink &sink,
                    cudaStream_t s) {
    if (rep <= 0) return KFB_OK;
    const bool tc = use_tc(prec, rep);
    if (dt == KFB_F64) return hessian_core<double>(s1, s2, rep, sigma, symmetric, tc, sink, s);
    return hessian_core<float>(s1, s2, rep, sigma, symmetric, tc, sink, s);
}

DerivSet dset(const void *x, const void *dx, const int32_t *q, const int32_t *n, int nm, int ma) {
    DerivSet d;
    d.x = x;
    d.dx = dx;
    d.v = view(q, n, nm, ma);
    return d;
}

}  // namespace

extern "C" {

const char *kfb_last_error(void) { return last_error(); }
int kfb_abi_version(void) { return KFB_ABI_VERSION; }

kfb_status kfb_set_timing(int enable) {
    set_timing(enable != 0);
    return KFB_OK;
}
double kfb_last_kernel_ms(void) { return last_kernel_ms(); }

kfb_status kfb_path_log_clear(void) {
    path_log_clear();
    return KFB_OK;
}

int kfb_path_log_read(char *buf, int len) {
    const std::string &s = path_log();
    if (buf && len > 0) {
        const int n = std::min<int>(len - 1, (int)s.size());
        std::memcpy(buf, s.data(), (size_t)n);
        buf[n] = '\0';
    }
    return (int)s.size();
}

kfb_status kfb_kernel_gaussian(const void *x1, const void *x2, const int32_t *q1,
                               const int32_t *q2, const int32_t *n1, const int32_t *n2, int nm1,
                               int nm2, int ma1, int ma2, int rep, double sigma, kfb_dtype x_dt,
                               kfb_precision prec, kfb_dtype out_dt, void *out, void *stream) {
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_prec(prec));
    KFB_TRY(check_set(x1, q1, n1, nm1, ma1, "set 1"));
    KFB_TRY(check_set(x2, q2, n2, nm2, ma2, "set 2"));
    cudaStream_t s = as_stream(stream);
    const size_t bytes = (size_t)nm1 * nm2 * esize(out_dt);
    if (bytes == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, bytes, s));
    ScalarProblem p;
    p.x1 = x1;
    p.x2 = x2;
    p.s1 = view(q1, n1, nm1, ma1);
    p.s2 = view(q2, n2, nm2, ma2);
    p.rep = rep;
    p.sigma = sigma;
    p.x_dt = x_dt;
    p.symmetric = false;
    PairSink sink;
    sink.out = out;
    sink.out_f64 = out_dt == KFB_F64;
    sink.mode = OUT_RECT;
    sink.n = nm2;
    return scalar_dispatch(p, prec, sink, s);
}

kfb_status kfb_kernel_gaussian_symm(const void *x, const int32_t *q, const int32_t *n, int nm,
                                    int ma, int rep, double sigma, kfb_dtype x_dt,
                                    kfb_precision prec, kfb_layout layout, kfb_dtype out_dt,
                                    void *out, void *stream) {
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_prec(prec));
    KFB_TRY(check_layout(layout));
    KFB_TRY(check_set(x, q, n, nm, ma, "set"));
    cudaStream_t s = as_stream(stream);
    const size_t count = layout == KFB_DENSE ? (size_t)nm * nm : (size_t)nm * (nm + 1) / 2;
    if (count == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, count * esize(out_dt), s));
    ScalarProblem p;
    p.x1 = p.x2 = x;
    p.s1 = p.s2 = view(q, n, nm, ma);
    p.rep = rep;
    p.sigma = sigma;
    p.x_dt = x_dt;
    p.symmetric = true;
    PairSink sink;
    sink.out = out;
    sink.out_f64 = out_dt == KFB_F64;
    sink.mode = OUT_SYMM;
    sink.layout = layout;
    sink.n = nm;
    return scalar_dispatch(p, prec, sink, s);
}

kfb_status kfb_kernel_gaussian_symm_host(const void *x_host, const int32_t *q, const int32_t *n,
                                         int nm, int ma, int rep, double sigma, kfb_dtype x_dt,
                                         kfb_precision prec, kfb_layout layout, kfb_dtype out_dt,
                                         void *out, void *stream) {
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_prec(prec));
    KFB_TRY(check_layout(layout));
    KFB_TRY(check_set(x_host, q, n, nm, ma, "set"));
    if (x_dt != KFB_F64 && x_dt != KFB_F32) return set_error(KFB_ERR_INVALID_ARG, "unknown dtype");
    cudaStream_t s = as_stream(stream);
    const size_t count = layout == KFB_DENSE ? (size_t)nm * nm : (size_t)nm * (nm + 1) / 2;
    if (count == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    if (prec != KFB_PREC_SPLIT_F16 || rep <= 0) {
        // no pipelined path for these: one copy, then the device-input kernel
        DevBuf xd;
        const size_t bytes = (size_t)nm * ma * (rep > 0 ? rep : 0) * esize(x_dt);
        KFB_TRY(xd.alloc(bytes, s));
        if (bytes)
            KFB_CUDA_TRY(cudaMemcpyAsync(xd.ptr, x_host, bytes, cudaMemcpyHostToDevice, s));
        KFB_TRY(kfb_kernel_gaussian_symm(xd.ptr, q, n, nm, ma, rep, sigma, x_dt, prec, layout,
                                         out_dt, out, stream));
        KFB_CUDA_TRY(cudaStreamSynchronize(s));
        return KFB_OK;
    }
    KFB_TRY(zero(out, count * esize(out_dt), s));
    ScalarProblem p;
    p.x1 = p.x2 = nullptr;
    p.s1 = p.s2 = view(q, n, nm, ma);
    p.rep = rep;
    p.sigma = sigma;
    p.x_dt = x_dt;
    p.symmetric = true;
    PairSink sink;
    sink.out = out;
    sink.out_f64 = out_dt == KFB_F64;
    sink.mode = OUT_SYMM;
    sink.layout = layout;
    sink.n = nm;
    return scalar_tc_from_host(p, x_host, sink, s);
}

kfb_status kfb_kernel_gaussian_jacobian(const void *x1, const void *x2, const void *dx2,
                                        const int32_t *q1, const int32_t *q2, const int32_t *n1,
                                        const int32_t *n2, int nm1, int nm2, int ma1, int ma2,
                                        int rep, int naq2, double sigma, kfb_dtype dt,
                                        kfb_precision prec, void *out, void *stream) {
    if (nm1 <= 0 || nm2 <= 0 || ma1 <= 0 || ma2 <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_deriv_prec(dt, prec));
    KFB_TRY(check_set(x1, q1, n1, nm1, ma1, "set 1"));
    KFB_TRY(check_set(x2, q2, n2, nm2, ma2, "set 2"));
    if (!dx2) return set_error(KFB_ERR_INVALID_ARG, "dX2 is null");
    KFB_TRY(naq_check(view(q2, n2, nm2, ma2), naq2, "naq2 != 3*sum(n2)"));
    cudaStream_t s = as_stream(stream);
    const size_t bytes = (size_t)nm1 * naq2 * esize(dt);
    if (bytes == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, bytes, s));
    ElemSink sink;
    sink.out = out;
    sink.f64 = dt == KFB_F64;
    sink.mode = EM_RECT;
    sink.ld = naq2;
    return jac_any(dt, prec, dset(x1, nullptr, q1, n1, nm1, ma1), dset(x2, dx2, q2, n2, nm2, ma2), rep,
                   sigma, 1.0, sink, s);
}

kfb_status kfb_kernel_gaussian_jacobian_t(const void *x1, const void *dx1, const void *x2,
                                          const int32_t *q1, const int32_t *q2,
                                          const int32_t *n1, const int32_t *n2, int nm1, int nm2,
                                          int ma1, int ma2, int rep, int naq1, double sigma,
                                          kfb_dtype dt, kfb_precision prec, void *out,
                                          void *stream) {
    if (nm1 <= 0 || nm2 <= 0 || ma1 <= 0 || ma2 <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_deriv_prec(dt, prec));
    KFB_TRY(check_set(x1, q1, n1, nm1, ma1, "set 1"));
    KFB_TRY(check_set(x2, q2, n2, nm2, ma2, "set 2"));
    if (!dx1) return set_error(KFB_ERR_INVALID_ARG, "dX1 is null");
    KFB_TRY(naq_check(view(q1, n1, nm1, ma1), naq1, "naq1 != 3*sum(n1)"));
    cudaStream_t s = as_stream(stream);
    const size_t bytes = (size_t)naq1 * nm2 * esize(dt);
    if (bytes == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, bytes, s));
    // G[b, off1[a] + c] = sum_{i in a} (sum_{j in b} w (x_j - x_i)) . J_i[:, c]
    //                   = -jacobian_t[off1[a] + c, b]
    ElemSink sink;
    sink.out = out;
    sink.f64 = dt == KFB_F64;
    sink.mode = EM_RECT_T;
    sink.ld = nm2;
    return jac_any(dt, prec, dset(x2, nullptr, q2, n2, nm2, ma2), dset(x1, dx1, q1, n1, nm1, ma1), rep,
                   sigma, -1.0, sink, s);
}

kfb_status kfb_kernel_gaussian_hessian(const void *x1, const void *dx1, const void *x2,
                                       const void *dx2, const int32_t *q1, const int32_t *q2,
                                       const int32_t *n1, const int32_t *n2, int nm1, int nm2,
                                       int ma1, int ma2, int rep, int naq1, int naq2,
                                       double sigma, kfb_dtype dt, kfb_precision prec,
                                       void *out, void *stream) {
    if (nm1 <= 0 || nm2 <= 0 || ma1 <= 0 || ma2 <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_deriv_prec(dt, prec));
    KFB_TRY(check_set(x1, q1, n1, nm1, ma1, "set 1"));
    KFB_TRY(check_set(x2, q2, n2, nm2, ma2, "set 2"));
    if (!dx1 || !dx2) return set_error(KFB_ERR_INVALID_ARG, "dX1/dX2 is null");
    KFB_TRY(naq_check(view(q1, n1, nm1, ma1), naq1, "naq1 != 3*sum(n1)"));
    KFB_TRY(naq_check(view(q2, n2, nm2, ma2), naq2, "naq2 != 3*sum(n2)"));
    cudaStream_t s = as_stream(stream);
    const size_t bytes = (size_t)naq1 * naq2 * esize(dt);
    if (bytes == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, bytes, s));
    ElemSink sink;
    sink.out = out;
    sink.f64 = dt == KFB_F64;
    sink.mode = EM_RECT;
    sink.ld = naq2;
    return hess_any(dt, prec, dset(x1, dx1, q1, n1, nm1, ma1), dset(x2, dx2, q2, n2, nm2, ma2), rep,
                    sigma, false, sink, s);
}

kfb_status kfb_kernel_gaussian_hessian_symm(const void *x, const void *dx, const int32_t *q,
                                            const int32_t *n, int nm, int ma, int rep, int naq,
                                            double sigma, kfb_dtype dt, kfb_precision prec,
                                            kfb_layout layout, void *out, void *stream) {
    if (nm <= 0 || ma <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "dims must be positive");
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_deriv_prec(dt, prec));
    KFB_TRY(check_layout(layout));
    KFB_TRY(check_set(x, q, n, nm, ma, "set"));
    if (!dx) return set_error(KFB_ERR_INVALID_ARG, "dX is null");
    KFB_TRY(naq_check(view(q, n, nm, ma), naq, "naq != 3*sum(n)"));
    cudaStream_t s = as_stream(stream);
    const size_t count = layout == KFB_DENSE ? (size_t)naq * naq : (size_t)naq * (naq + 1) / 2;
    if (count == 0) return KFB_OK;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, count * esize(dt), s));
    ElemSink sink;
    sink.out = out;
    sink.f64 = dt == KFB_F64;
    sink.mode = EM_SYM;
    sink.layout = layout == KFB_DENSE ? LAYOUT_DENSE_LOWER : layout;
    sink.ld = naq;
    DerivSet d = dset(x, dx, q, n, nm, ma);
    return hess_any(dt, prec, d, d, rep, sigma, true, sink, s);
}

kfb_status kfb_kernel_gaussian_full(const void *x1, const void *dx1, const void *x2,
                                    const void *dx2, const int32_t *q1, const int32_t *q2,
                                    const int32_t *n1, const int32_t *n2, int nm1, int nm2,
                                    int ma1, int ma2, int rep, int naq1, int naq2, double sigma,
                                    kfb_dtype dt, kfb_precision prec, void *out, void *stream) {
    if (nm1 <= 0 || nm2 <= 0 || ma1 <= 0 || ma2 <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_deriv_prec(dt, prec));
    KFB_TRY(check_set(x1, q1, n1, nm1, ma1, "set 1"));
    KFB_TRY(check_set(x2, q2, n2, nm2, ma2, "set 2"));
    if (!dx1 || !dx2) return set_error(KFB_ERR_INVALID_ARG, "dX1/dX2 is null");
    KFB_TRY(naq_check(view(q1, n1, nm1, ma1), naq1, "naq1 != 3*sum(n1)"));
    KFB_TRY(naq_check(view(q2, n2, nm2, ma2), naq2, "naq2 != 3*sum(n2)"));
    cudaStream_t s = as_stream(stream);
    const long long R = (long long)nm1 + naq1, C = (long long)nm2 + naq2;
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, (size_t)(R * C) * esize(dt), s));
    // scalar block [0:nm1, 0:nm2]
    ScalarProblem p;
    p.x1 = x1;
    p.x2 = x2;
    p.s1 = view(q1, n1, nm1, ma1);
    p.s2 = view(q2, n2, nm2, ma2);
    p.rep = rep;
    p.sigma = sigma;
    p.x_dt = dt;
    PairSink ps;
    ps.out = out;
    ps.out_f64 = dt == KFB_F64;
    ps.mode = OUT_RECT;
    ps.n = C;
    KFB_TRY(scalar_dispatch(p, prec, ps, s));
    const DerivSet d1 = dset(x1, dx1, q1, n1, nm1, ma1), d2 = dset(x2, dx2, q2, n2, nm2, ma2);
    // [0:nm1, nm2:] = +jacobian(X1, X2, dX2)
    ElemSink sj;
    sj.out = out;
    sj.f64 = dt == KFB_F64;
    sj.mode = EM_RECT;
    sj.ld = C;
    sj.col_base = nm2;
    KFB_TRY(jac_any(dt, prec, d1, d2, rep, sigma, 1.0, sj, s));
    // [nm1:, 0:nm2] = -jacobian_t(X1, dX1, X2) = G^T with G from (outer 2, inner 1)
    ElemSink st;
    st.out = out;
    st.f64 = dt == KFB_F64;
    st.mode = EM_RECT_T;
    st.ld = C;
    st.col_base = nm1;
    KFB_TRY(jac_any(dt, prec, d2, d1, rep, sigma, 1.0, st, s));
    // [nm1:, nm2:] = hessian
    ElemSink sh;
    sh.out = out;
    sh.f64 = dt == KFB_F64;
    sh.mode = EM_RECT;
    sh.ld = C;
    sh.row_base = nm1;
    sh.col_base = nm2;
    return hess_any(dt, prec, d1, d2, rep, sigma, false, sh, s);
}

kfb_status kfb_kernel_gaussian_full_symm(const void *x, const void *dx, const int32_t *q,
                                         const int32_t *n, int nm, int ma, int rep, int naq,
                                         double sigma, kfb_dtype dt, kfb_precision prec,
                                         kfb_layout layout, void *out, void *stream) {
    if (nm <= 0 || ma <= 0 || rep <= 0)
        return set_error(KFB_ERR_INVALID_ARG, "dims must be positive");
    KFB_TRY(check_sigma(sigma));
    KFB_TRY(check_deriv_prec(dt, prec));
    KFB_TRY(check_layout(layout));
    KFB_TRY(check_set(x, q, n, nm, ma, "set"));
    if (!dx) return set_error(KFB_ERR_INVALID_ARG, "dX is null");
    KFB_TRY(naq_check(view(q, n, nm, ma), naq, "naq != 3*sum(n)"));
    cudaStream_t s = as_stream(stream);
    const long long big = (long long)nm + naq;
    const size_t count = layout == KFB_DENSE ? (size_t)(big * big) : (size_t)(big * (big + 1) / 2);
    if (!out) return set_error(KFB_ERR_INVALID_ARG, "out is null");
    KFB_TRY(zero(out, count * esize(dt), s));
    ScalarProblem p;
    p.x1 = p.x2 = x;
    p.s1 = p.s2 = view(q, n, nm, ma);
    p.rep = rep;
    p.sigma = sigma;
    p.x_dt = dt;
    p.symmetric = true;
    PairSink ps;
    ps.out = out;
    ps.out_f64 = dt == KFB_F64;
    ps.mode = OUT_SYMM;
    ps.layout = layout;
    ps.n = big;
    {
        TraceScope tr("full_symm:scalar", s);
        KFB_TRY(scalar_dispatch(p, prec, ps, s));
    }
    const DerivSet d = dset(x, dx, q, n, nm, ma);
    // jacobian block at rows [0, nm), columns [nm, big) and its mirror
    ElemSink sj;
    sj.out = out;
    sj.f64 = dt == KFB_F64;
    sj.mode = EM_SYM;
    sj.layout = layout;
    sj.ld = big;
    sj.col_base = nm;
    {
        TraceScope tr("full_symm:jacobian", s);
        KFB_TRY(jac_any(dt, prec, d, d, rep, sigma, 1.0, sj, s));
    }
    ElemSink sh;
    sh.out = out;
    sh.f64 = dt == KFB_F64;
    sh.mode = EM_SYM;
    sh.layout = layout;
    sh.ld = big;
    sh.row_base = nm;
    sh.col_base = nm;
    TraceScope tr("full_symm:hessian", s);
    return hess_any(dt, prec, d, d, rep, sigma, true, sh, s);
}

kfb_status kfb_full_to_rfp(const void *a, int n, kfb_layout uplo, kfb_dtype dt, void *arf,
                           void *stream) {
    if (n < 0 || (uplo != KFB_RFP_U && uplo != KFB_RFP_L))
        return set_error(KFB_ERR_INVALID_ARG, "full_to_rfp: bad n or uplo");
    return full_to_rfp(a, n, uplo, dt, arf, as_stream(stream));
}

kfb_status kfb_rfp_to_full(const void *arf, int n, kfb_layout uplo, kfb_dtype dt, void *a,
                           void *stream) {
    if (n < 0 || (uplo != KFB_RFP_U && uplo != KFB_RFP_L))
        return set_error(KFB_ERR_INVALID_ARG, "rfp_to_full: bad n or uplo");
    return rfp_to_full(arf, n, uplo, dt, a, as_stream(stream));
}

kfb_status kfb_rfp_add_diag(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt,
                            void *stream) {
    if (n < 0 || (uplo != KFB_RFP_U && uplo != KFB_RFP_L))
        return set_error(KFB_ERR_INVALID_ARG, "rfp_add_diag: bad n or uplo");
    return rfp_add_diag(arf, n, l2, uplo, dt, as_stream(stream));
}

kfb_status kfb_rfp_potrf(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt, int *info,
                         void *stream) {
    if (n < 0 || !info || (uplo != KFB_RFP_U && uplo != KFB_RFP_L))
        return set_error(KFB_ERR_INVALID_ARG, "rfp_potrf: bad argument");
    return rfp_potrf(arf, n, l2, uplo, dt, info, as_stream(stream));
}

kfb_status kfb_rfp_potrs(const void *arf, void *b, int n, int nrhs, kfb_layout uplo,
                         kfb_dtype dt, void *stream) {
    if (n < 0 || nrhs < 0 || (uplo != KFB_RFP_U && uplo != KFB_RFP_L))
        return set_error(KFB_ERR_INVALID_ARG, "rfp_potrs: bad argument");
    return rfp_potrs(arf, b, n, nrhs, uplo, dt, as_stream(stream));
}

kfb_status kfb_cho_solve_rfp(void *arf, const double *y, int n, double l2, kfb_layout uplo,
                             double *alpha, int *info, void *stream) {
    if (n <= 0) return set_error(KFB_ERR_INVALID_ARG, "n must be > 0");
    if (!arf || !y || !alpha || !info) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (uplo != KFB_RFP_U && uplo != KFB_RFP_L)
        return set_error(KFB_ERR_INVALID_ARG, "uplo must be 'U' or 'L'");
    cudaStream_t s = as_stream(stream);
    KFB_TRY(cho_solve_rfp_f64(static_cast<double *>(arf), y, n, l2, uplo, alpha, info, s));
    if (*info != 0) return set_error(KFB_ERR_NOT_PD, "DPFTRF failed, info=%d", *info);
    return KFB_OK;
}

kfb_status kfb_krr_solve_mixed(const float *k_rfp, const double *y, int n, double l2,
                               kfb_layout uplo, double tol, int maxit, int flags, double *alpha,
                               kfb_solve_info *info, void *stream) {
    if (n <= 0) return set_error(KFB_ERR_INVALID_ARG, "n must be > 0");
    if (!k_rfp || !y || !alpha) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (uplo != KFB_RFP_U && uplo != KFB_RFP_L)
        return set_error(KFB_ERR_INVALID_ARG, "uplo must be RFP");
    if (!(tol > 0.0) || maxit < 0) return set_error(KFB_ERR_INVALID_ARG, "bad tol / maxit");
    return krr_solve_mixed(k_rfp, y, n, l2, uplo, tol, maxit, flags, alpha, info,
                           as_stream(stream));
}

kfb_status kfb_feature_gramian(const float *z, const double *y, int nm, int d, kfb_layout layout,
                               float *ztz, double *zty, void *stream) {
    if (nm <= 0 || d <= 0) return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    if (!z || !ztz || (y && !zty)) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (layout != KFB_DENSE && layout != KFB_RFP_U && layout != KFB_RFP_L)
        return set_error(KFB_ERR_INVALID_ARG, "layout must be dense or RFP");
    return feature_gramian(z, y, nm, d, layout, ztz, zty, as_stream(stream));
}

kfb_status kfb_ridge_solve_mixed(const float *z, const double *y, int nm, int d, double l2,
                                 double tol, int maxit, int flags, double *w,
                                 kfb_solve_info *info, void *stream) {
    if (nm <= 0 || d <= 0) return set_error(KFB_ERR_INVALID_ARG, "All dims must be positive.");
    if (!z || !y || !w) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (!(tol > 0.0) || maxit < 0 || !(l2 >= 0.0))
        return set_error(KFB_ERR_INVALID_ARG, "bad l2 / tol / maxit");
    return ridge_solve_mixed(z, y, nm, d, l2, tol, maxit, flags, w, info, as_stream(stream));
}

}  // extern "C"
