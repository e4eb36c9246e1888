/*
 * kfb.h -- C ABI of the B200-native FCHL19 local-kernel / RFP-Cholesky library
 * (libkfb.so).
 *
 * Every entry point replaces one routine of the reference's pybind11 modules
 * kernelforge.local_kernels, kernelforge.kernelmath,
 * kernelforge.cuda_local_kernels and kernelforge.cuda_global_kernels; the
 * replaced interface is cited (reference file:line) above each declaration.
 *
 * Memory and argument conventions (shared by all calls):
 *   - X / dX / outputs / RFP arrays / right-hand sides are DEVICE pointers.
 *     X is (nm, ma, rep), dX is (nm, ma, rep, 3*ma), both C-contiguous; the
 *     element type is given by a kfb_dtype argument.
 *   - Q (nm, ma) and N (nm,) are HOST int32 pointers: the atom bucketing by
 *     label (nuclear charge) is planned on the host, exactly as the reference
 *     reads its labels on the host (src/local_kernels.cpp:31-149).
 *   - N is clamped to [0, ma]; padded atoms are ignored.
 *   - naq = 3 * sum(clamp(N)) (derivative axis length).
 *   - Work is enqueued on `stream` (a cudaStream_t, NULL = legacy default
 *     stream); the call returns once the work is enqueued, except where a host
 *     result is returned (info codes, iteration counts), which synchronises
 *     the stream.
 *   - Scratch memory is taken from the device's stream-ordered pool
 *     (cudaMallocAsync) and released on the same stream.
 *   - Errors are returned, never abort()ed; kfb_last_error() gives the message
 *     of the calling thread's last failure.
 */
#ifndef KFB_H
#define KFB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define KFB_ABI_VERSION 1

typedef enum kfb_status {
    KFB_OK = 0,
    KFB_ERR_INVALID_ARG = 1,    /* reference: std::invalid_argument -> ValueError */
    KFB_ERR_NOT_PD = 2,         /* Cholesky info > 0 (leading minor not positive) */
    KFB_ERR_ALLOC = 3,          /* device allocation failed */
    KFB_ERR_CUDA = 4,           /* CUDA / cuBLAS error */
    KFB_ERR_TIMEOUT = 5,        /* a bounded device-side wait gave up */
    KFB_ERR_NO_CONVERGENCE = 6, /* iterative refinement missed its tolerance */
    KFB_ERR_UNSUPPORTED = 7     /* device or configuration not supported */
} kfb_status;

typedef enum kfb_dtype { KFB_F32 = 0, KFB_F64 = 1 } kfb_dtype;

/* Arithmetic of the distance contraction ||x_i - x_j||^2. */
typedef enum kfb_precision {
    KFB_PREC_FP64 = 0,      /* FP64 CUDA cores (the plain FP64 GPU path)           */
    KFB_PREC_FP32 = 1,      /* FP32 CUDA cores                                      */
    KFB_PREC_SPLIT_F16 = 2  /* tcgen05 tensor cores: x = hi + lo (fp16 pair),
                               hi*hi + hi*lo + lo*hi with FP32 accumulation in TMEM */
} kfb_precision;

/* Output storage of a symmetric matrix. */
typedef enum kfb_layout {
    KFB_DENSE = 0,  /* full (n, n) row-major                                        */
    KFB_RFP_U = 1,  /* RFP, TRANSR='N', Fortran UPLO='U' (the CPU modules' packing) */
    KFB_RFP_L = 2   /* RFP, TRANSR='N', Fortran UPLO='L' (the GPU modules' packing) */
} kfb_layout;

const char *kfb_last_error(void);
int kfb_abi_version(void);

/* Tracing.  When enabled, each call brackets its main tile kernel (the tensor-
 * core or CUDA-core tile kernel of the scalar kernels) with CUDA events on the
 * caller's stream and keeps the elapsed time, read back by
 * kfb_last_kernel_ms() (milliseconds; the call synchronises the stream).
 * No reference counterpart: the reference prints always-on stage timers to
 * stderr (src/cuda_local_kernels.cu:1902-1909). */
kfb_status kfb_set_timing(int enable);
double kfb_last_kernel_ms(void);

/* Code-path log of the calling thread.  Where a call chooses between several
 * implementations of one step (the Hessian's CUDA-core t' kernel, its GEMM form
 * with the rank term inside Y, or the separate rank kernel), it appends the
 * name of the path it took; kfb_path_log_read copies the comma-separated log
 * (NUL-terminated, truncated to len - 1 characters) and returns its full
 * length.  No reference counterpart (the reference has one path per call). */
kfb_status kfb_path_log_clear(void);
int kfb_path_log_read(char *buf, int len);

/* ---------------------------------------------------------------------- */
/* Scalar kernels: K[a,b] = sum_{i in a, j in b, q_i = q_j}                */
/*                          exp(-||x_i - x_j||^2 / (2 sigma^2))            */
/* ---------------------------------------------------------------------- */

/* K (nm1, nm2) row-major, element type `out_dt`.
 * Replaces local_kernels.kernel_gaussian (src/local_kernels_bindings.cpp:28-104,
 * src/local_kernels.cpp:155-298) and cuda_local_kernels.kernel_gaussian_rect
 * (src/cuda_local_kernels_bindings.cpp:845-851). */
kfb_status kfb_kernel_gaussian(const void *x1, const void *x2, const int32_t *q1,
                               const int32_t *q2, const int32_t *n1, const int32_t *n2,
                               int nm1, int nm2, int ma1, int ma2, int rep, double sigma,
                               kfb_dtype x_dt, kfb_precision prec, kfb_dtype out_dt, void *out,
                               void *stream);

/* Symmetric kernel; layout KFB_DENSE fills both triangles of (nm, nm),
 * KFB_RFP_U / KFB_RFP_L write nm*(nm+1)/2 packed entries.
 * Replaces local_kernels.kernel_gaussian_symm / _symm_rfp
 * (src/local_kernels.cpp:584-758, :403-577) and
 * cuda_local_kernels.kernel_gaussian_symm / _symm_rfp
 * (src/cuda_local_kernels.cu:2989-3131, :3224-3359). */
kfb_status kfb_kernel_gaussian_symm(const void *x, const int32_t *q, const int32_t *n, int nm,
                                    int ma, int rep, double sigma, kfb_dtype x_dt,
                                    kfb_precision prec, kfb_layout layout, kfb_dtype out_dt,
                                    void *out, void *stream);

/* kfb_kernel_gaussian_symm with X (nm, ma, rep) in HOST memory (page-locked
 * for overlap) and `out` on the device.  With KFB_PREC_SPLIT_F16 the copy of
 * X runs in chunks of molecules (KFB_H2D_CHUNKS, default 8) while the tensor
 * cores work on the tiles whose molecules have arrived; each label is centred
 * on the mean of its rows in the first chunk holding it, so the values differ
 * from the device-input call at the split's rounding level.  Other
 * precisions copy X once and run the device-input kernel.  Returns after the
 * kernel has finished (the host buffer may be reused). */
kfb_status kfb_kernel_gaussian_symm_host(const void *x_host, const int32_t *q, const int32_t *n,
                                         int nm, int ma, int rep, double sigma, kfb_dtype x_dt,
                                         kfb_precision prec, kfb_layout layout, kfb_dtype out_dt,
                                         void *out, void *stream);

/* ---------------------------------------------------------------------- */
/* Derivative kernels (element type of x, dx and out: `dt`)                */
/* ---------------------------------------------------------------------- */

/* K (nm1, naq2): +dK/dR2.  Replaces local_kernels.kernel_gaussian_jacobian
 * (src/local_kernels_bindings.cpp:158-270, src/local_kernels.cpp:791-974). */
kfb_status kfb_kernel_gaussian_jacobian(const void *x1, const void *x2, const void *dx2,
                                        const int32_t *q1, const int32_t *q2, const int32_t *n1,
                                        const int32_t *n2, int nm1, int nm2, int ma1, int ma2,
                                        int rep, int naq2, double sigma, kfb_dtype dt,
                                        kfb_precision prec, void *out, void *stream);

/* K (naq1, nm2): +dK/dR1.  Replaces local_kernels.kernel_gaussian_jacobian_t
 * (src/local_kernels_bindings.cpp:272-386, src/local_kernels.cpp:991-1166). */
kfb_status kfb_kernel_gaussian_jacobian_t(const void *x1, const void *dx1, const void *x2,
                                          const int32_t *q1, const int32_t *q2,
                                          const int32_t *n1, const int32_t *n2, int nm1, int nm2,
                                          int ma1, int ma2, int rep, int naq1, double sigma,
                                          kfb_dtype dt, kfb_precision prec, void *out,
                                          void *stream);

/* H (naq1, naq2).  Replaces local_kernels.kernel_gaussian_hessian
 * (src/local_kernels_bindings.cpp:388-525, src/local_kernels.cpp:1171-1419). */
kfb_status kfb_kernel_gaussian_hessian(const void *x1, const void *dx1, const void *x2,
                                       const void *dx2, const int32_t *q1, const int32_t *q2,
                                       const int32_t *n1, const int32_t *n2, int nm1, int nm2,
                                       int ma1, int ma2, int rep, int naq1, int naq2,
                                       double sigma, kfb_dtype dt, kfb_precision prec,
                                       void *out, void *stream);

/* Symmetric Hessian.  KFB_DENSE: (naq, naq) with only the lower triangle
 * filled (upper triangle zero), as kernel_gaussian_hessian_symm
 * (src/local_kernels.cpp:1421-1655); KFB_RFP_U / KFB_RFP_L: packed, as
 * kernel_gaussian_hessian_symm_rfp (src/local_kernels.cpp:1664-1900). */
kfb_status kfb_kernel_gaussian_hessian_symm(const void *x, const void *dx, const int32_t *q,
                                            const int32_t *n, int nm, int ma, int rep, int naq,
                                            double sigma, kfb_dtype dt, kfb_precision prec,
                                            kfb_layout layout, void *out, void *stream);

/* Full energy+force kernel ((nm1+naq1), (nm2+naq2)); blocks [scalar, +jacobian;
 * -jacobian_t, hessian].  Replaces local_kernels.kernel_gaussian_full
 * (src/local_kernels.cpp:1918-2188). */
kfb_status kfb_kernel_gaussian_full(const void *x1, const void *dx1, const void *x2,
                                    const void *dx2, const int32_t *q1, const int32_t *q2,
                                    const int32_t *n1, const int32_t *n2, int nm1, int nm2,
                                    int ma1, int ma2, int rep, int naq1, int naq2, double sigma,
                                    kfb_dtype dt, kfb_precision prec, void *out, void *stream);

/* Symmetric full kernel of order BIG = nm + naq; KFB_DENSE is fully filled.
 * Replaces local_kernels.kernel_gaussian_full_symm / _full_symm_rfp
 * (src/local_kernels.cpp:2201-2498, :2511-2815) and
 * cuda_local_kernels.kernel_gaussian_full_symm / _full_symm_rfp
 * (src/cuda_local_kernels.cu:1871-2342, :3657-4097). */
kfb_status kfb_kernel_gaussian_full_symm(const void *x, const void *dx, const int32_t *q,
                                         const int32_t *n, int nm, int ma, int rep, int naq,
                                         double sigma, kfb_dtype dt, kfb_precision prec,
                                         kfb_layout layout, void *out, void *stream);

/* ---------------------------------------------------------------------- */
/* FP64-class products on the int8 tensor cores                            */
/* ---------------------------------------------------------------------- */

/* C (m, n) = alpha A B^T (beta = 0) or C + alpha A B^T (beta = 1) for
 * row-major FP64 A (m, k; lda), B (n, k; ldb), C (m, n; ldc).  Each row of A
 * and B is cut into `slices` (2..7) planes of balanced base-128 int8 digits
 * under a per-row power-of-two scale; the digit-plane products are exact int32
 * sums on the int8 tensor cores (tcgen05 kind::i8) and are combined in FP64,
 * so each operand keeps about 7 * slices - 1 significant bits (slices = 7:
 * |error| <~ 2^-47 k max|A_i| max|B_j|).  k <= 65536.  Allocates scratch.
 * No reference counterpart: the reference's FP64 products are BLAS dgemm calls
 * (src/local_kernels.cpp:237,689,940,1394,2751,3053-3107). */
kfb_status kfb_gemm_f64_i8(int m, int n, int k, double alpha, const double *a, int lda,
                           const double *b, int ldb, double beta, double *c, int ldc, int slices,
                           void *stream);

/* ---------------------------------------------------------------------- */
/* RFP storage and the Cholesky solve                                      */
/* ---------------------------------------------------------------------- */

/* Symmetric dense (n, n) <-> RFP.  Replaces kernelmath.full_to_rfp /
 * rfp_to_full (src/math_bindings.cpp:85-180, src/math.cpp:173-211). */
kfb_status kfb_full_to_rfp(const void *a, int n, kfb_layout uplo, kfb_dtype dt, void *arf,
                           void *stream);
kfb_status kfb_rfp_to_full(const void *arf, int n, kfb_layout uplo, kfb_dtype dt, void *a,
                           void *stream);

/* arf[diag(i)] += l2.  Replaces add_l2_diag_rfp_kernel / _upper_kernel
 * (src/cuda_global_kernels.cu:436-475). */
kfb_status kfb_rfp_add_diag(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt,
                            void *stream);

/* In-place Cholesky of an RFP matrix after adding l2 to its diagonal; *info is
 * 0 or the order of the first non-positive leading minor (synchronises).
 * Replaces cuda_global_kernels.rfp_potrf (src/cuda_global_kernels.cu:847-868,
 * src/curfp_spftrf.cpp:182-292) for F32 and LAPACK dpftrf for F64. */
kfb_status kfb_rfp_potrf(void *arf, int n, double l2, kfb_layout uplo, kfb_dtype dt, int *info,
                         void *stream);

/* Solve with the factor from kfb_rfp_potrf; B is (n, nrhs) column-major
 * (ldb = n), overwritten with X.  Replaces cuda_global_kernels.rfp_potrs
 * (src/cuda_global_kernels.cu:880-893, src/curfp_spftrs.cpp:215-302). */
kfb_status kfb_rfp_potrs(const void *arf, void *b, int n, int nrhs, kfb_layout uplo,
                         kfb_dtype dt, void *stream);

/* FP64 (K + l2 I) alpha = y, K in FP64 RFP (overwritten with the factor);
 * *info as LAPACK.  Replaces kernelmath.cho_solve_rfp
 * (src/math_bindings.cpp:49-76, src/math.cpp:134-171). */
kfb_status kfb_cho_solve_rfp(void *arf, const double *y, int n, double l2, kfb_layout uplo,
                             double *alpha, int *info, void *stream);

/* Mixed-precision KRR solve: (K + l2 I) alpha = y with K given as an FP32 RFP
 * array (not modified).  The factor is this library's tensor-core Cholesky of
 * the dense lower triangle of K + (l2 + shift) I: FP32-class by default (K's
 * dominant eigenpair deflated, 4 digit planes of 7 bits in the int8 trailing
 * updates, FP32 diagonal blocks) or FP64-class with KFB_SOLVE_FP64_FACTOR (6
 * planes, FP64 diagonal blocks, no deflation); residuals, corrections and
 * norms are FP64 (conjugate-gradient refinement preconditioned by the
 * factor).  Stops at ||r|| <= tol * ||y||; KFB_ERR_NOT_PD if K + l2 I is
 * indefinite at FP32 storage precision (unless KFB_SOLVE_LAMBDA_FLOOR).
 * No reference counterpart: it replaces the reference's FP32 rfp_potrf +
 * rfp_potrs pair and its CPU FP64 fallback (models/cuda_local_krr.py:640-675). */
typedef struct kfb_solve_info {
    int iterations;       /* refinement (CG) iterations taken              */
    int factor_info;      /* potrf info of the last factorisation tried    */
    double shift;         /* diagonal shift added to the FP32 factor only  */
    double rel_residual;  /* final ||y - (K + l2_eff I) alpha|| / ||y||  */
    int used_cg;          /* 1 if CG refinement ran                        */
    double lambda_eff;    /* regularisation of the system solved           */
} kfb_solve_info;

/* flags of kfb_krr_solve_mixed */
#define KFB_SOLVE_LAMBDA_FLOOR 1  /* if K + l2 I is indefinite at FP32 storage
                                     precision, raise l2 (x10 steps) until it is
                                     not, and report it in lambda_eff */
#define KFB_SOLVE_FP64_FACTOR 2   /* FP64-class factor instead of FP32-class;
                                     the refinement then converges in one or
                                     two steps */

kfb_status kfb_krr_solve_mixed(const float *k_rfp, const double *y, int n, double l2,
                               kfb_layout uplo, double tol, int maxit, int flags,
                               double *alpha, kfb_solve_info *info, void *stream);

/* ---------------------------------------------------------------------- */
/* Feature maps summed per molecule and their normal equations             */
/* ---------------------------------------------------------------------- */

/* Element-stratified random Fourier features, summed per molecule:
 *   z[m][:] = sum over atoms a of molecule m: sqrt(2/d) cos(x_a . w[e_a] + b[e_a])
 * q (nm, ma) HOST int32 element INDICES (0 .. nelem-1, -1 = padding, unlike
 * the nuclear charges of the kernels above); w (nelem, rep, d) and b (nelem, d)
 * device float32; z (nm, d) device float32, overwritten.  x . w runs on the
 * tensor cores as split-fp16 products (FP32-class accuracy); rep % 16 == 0.
 * Replaces rff_features_elemental_cuda (src/cuda_rff_features.hpp:47-53, bound
 * in src/cuda_rff_features_bindings.cpp:70-80) and the CPU
 * kf::rff::rff_features_elemental (src/rff_elemental.hpp:20-24). */
kfb_status kfb_rff_features_elemental(const void *x, const int32_t *q, const int32_t *n, int nm,
                                      int ma, int rep, const float *w, const float *b, int nelem,
                                      int d, kfb_dtype x_dt, float *z, void *stream);

/* Force features of the elemental RFF model: g (naq, d) device float32, row
 * 3 off_m + 3 a + t = sqrt(2/d) sum_j sin(x_j W[e_j] + b[e_j]) (W[e_j]^T dX[m, j, :, 3 a + t])
 * over the atoms j of molecule m, so that forces are F = g w.  x (nm, ma, rep) and
 * dx (nm, ma, rep, 3 ma) device of type x_dt; q (element index, -1 = padding) and n
 * host; w (nelem, rep, d), b (nelem, d) device float32; d a multiple of 8.  Tensor
 * cores (split fp16, FP32 accumulation): the pre-activations, then the Jacobian rows
 * times W with the sin weights and the per-molecule sums in the GEMM epilogue.
 * Replaces rff_gradient_elemental_cuda (src/cuda_rff_features.hpp:55-63, the
 * transpose of the CPU kf::rff::rff_gradient_elemental, src/rff_elemental.cpp:363-500). */
kfb_status kfb_rff_gradient_elemental(const void *x, const void *dx, const int32_t *q,
                                      const int32_t *n, int nm, int ma, int rep, const float *w,
                                      const float *b, int nelem, int d, kfb_dtype x_dt, float *g,
                                      void *stream);

/* Normal equations of a linear ridge model on per-molecule features:
 * ztz = Z^T Z (d x d; KFB_DENSE both triangles, or RFP), zty = Z^T y (float64;
 * skipped when y is NULL).  z (nm, d) device float32, y (nm,) device float64.
 * FP32 SYRK without reduced-precision shortcuts.  Replaces the Gramian half of
 * rff_gramian_elemental_rfp_cuda (src/cuda_rff_features.hpp:85-93; SSFRK +
 * SGEMV in src/cuda_rff_features.cu:1602-1670). */
kfb_status kfb_feature_gramian(const float *z, const double *y, int nm, int d, kfb_layout layout,
                               float *ztz, double *zty, void *stream);

/* Linear ridge weights on per-molecule features: (Z^T Z + l2 I) w = Z^T y,
 * z (nm, d) device float32, y (nm,) device float64, w (d,) device float64.
 * FP32 factor of the normal equations formed from Z with its dominant
 * direction projected out (and restored by a Sherman-Morrison term), FP64
 * conjugate-gradient refinement against the exact operator Z^T (Z w) applied
 * from Z; stops at ||r|| <= tol ||Z^T y||.  Flags and info as for
 * kfb_krr_solve_mixed.  Replaces the FP32 normal-equation solve of
 * models/cuda_local_rff.py:684-712 (rfp_potrf / rfp_potrs on Z^T Z). */
kfb_status kfb_ridge_solve_mixed(const float *z, const double *y, int nm, int d, double l2,
                                 double tol, int maxit, int flags, double *w,
                                 kfb_solve_info *info, void *stream);

/* Exact local-kernel values of atom pairs, the training targets of the learned
 * map: out[p] = exp(-|x[pi[p]] - x[pj[p]]|^2 / (2 sigma^2)), x (nrows, rep)
 * device, pi / pj device int32 row indices (an index outside [0, nrows) gives
 * KFB_ERR_INVALID_ARG; the kernel checks every index).  The pair term of the scalar
 * kernel (src/local_kernels.cpp:276-285). */
kfb_status kfb_pair_gaussian(const void *x, long long nrows, const int32_t *pi,
                             const int32_t *pj, int npairs, int rep, double sigma, kfb_dtype x_dt,
                             float *out, void *stream);

/* Learned cos-MLP feature map (no counterpart in the reference; it stands in
 * for the random Fourier features above).  Per element e:
 *   phi_e(x) = sqrt(2/d) cos(W2_e cos(W1_e x + b1_e) + b2_e)
 * W1 (nelem, hidden, rep), b1 (nelem, hidden), W2 (nelem, d, hidden),
 * b2 (nelem, d): FP32 master copies on the device, BF16 copies feed the tensor
 * cores (FP32 accumulation).  The handle owns parameters, Adam state and the
 * workspace of batches of up to max_pairs atom pairs. */
typedef struct kfb_cosmlp kfb_cosmlp;

kfb_status kfb_cosmlp_create(int nelem, int rep, int hidden, int d, int max_pairs,
                             kfb_cosmlp **out);
void kfb_cosmlp_destroy(kfb_cosmlp *h);
/* Device pointers to the FP32 parameters (write them, then kfb_cosmlp_sync). */
kfb_status kfb_cosmlp_params(kfb_cosmlp *h, float **w1, float **b1, float **w2, float **b2);
/* Device pointers to the gradients of the last pair step (one element's
 * tensors: (hidden, rep), (hidden,), (d, hidden), (d,)). */
kfb_status kfb_cosmlp_grads(kfb_cosmlp *h, float **w1, float **b1, float **w2, float **b2);
/* Refresh the BF16 copies from the FP32 parameters; optionally zero the Adam
 * moments and step counts. */
kfb_status kfb_cosmlp_sync(kfb_cosmlp *h, int reset_optimizer, void *stream);
/* Adam state for checkpoints: m[4], v[4] device pointers (same shapes as the
 * parameters), steps[nelem] host copy of the per-element step counts. */
kfb_status kfb_cosmlp_optimizer_state(kfb_cosmlp *h, float **m, float **v, int *steps);
kfb_status kfb_cosmlp_set_steps(kfb_cosmlp *h, const int *steps);
/* One training step of element elem on npairs pairs: rows pi[p], pj[p] of x
 * (nrows, rep) device, target (npairs,) device float32; an index outside
 * [0, nrows) gives KFB_ERR_INVALID_ARG (the gather checks every index).  Loss
 * mean_p (phi(x_i) . phi(x_j) - target_p)^2 (returned in *loss when not NULL);
 * gradients are left in the handle; update != 0 applies an Adam step
 * (beta 0.9 / 0.999, eps 1e-8) with learning rate lr.  Synchronises the stream. */
kfb_status kfb_cosmlp_pair_step(kfb_cosmlp *h, int elem, const void *x, long long nrows,
                                kfb_dtype x_dt, const int32_t *pi, const int32_t *pj,
                                const float *target, int npairs, float lr, int update,
                                double *loss, void *stream);
/* Learned features summed per molecule, the analogue of
 * kfb_rff_features_elemental (same x / q / n conventions): z (nm, d) float32. */
kfb_status kfb_cosmlp_features_elemental(kfb_cosmlp *h, const void *x, const int32_t *q,
                                         const int32_t *n, int nm, int ma, int rep,
                                         kfb_dtype x_dt, float *z, void *stream);

/* ---------------------------------------------------------------------- */
/* Contracted energy / force prediction (the "J^T alpha" form)             */
/* ---------------------------------------------------------------------- */

/* alpha_desc (nm2, ma2, rep) double: alpha_desc[b, j] = dX2[b, j] (rep x 3 n_b)
 * times alpha[off_b : off_b + 3 n_b] (off_b = 3 sum_{b' < b} n_b'), zero for
 * padded atoms; dx2 (nm2, ma2, rep, 3 ma2) of element type x_dt, alpha (naq2,)
 * double.  n2 host; q2 (host) may be NULL: the contraction does not depend
 * on the labels.  Replaces
 * local_kernels.kernel_gaussian_local_compute_alpha_desc
 * (src/local_kernels_bindings.cpp:1179-1243, src/local_kernels.cpp:2821-2894). */
kfb_status kfb_local_alpha_desc(const void *dx2, const int32_t *q2, const int32_t *n2, int nm2,
                                int ma2, int rep, kfb_dtype x_dt, const double *alpha,
                                double *alpha_desc, void *stream);

/* Predictions of a model with coefficients [alpha_E; alpha_F] over the
 * training set (x2, alpha_desc = kfb_local_alpha_desc of alpha_F) at the query
 * set (x1, dx1), without forming the E+F kernel matrix:
 *   e_out (nm1,)  = rows of kernel_gaussian_full(query, training) for the
 *                   energies times [alpha_E; alpha_F],
 *   f_out (naq1,) = the force rows (naq1 = 3 sum n1) times the same vector.
 * alpha_e NULL drops the alpha_E terms: e_out is then
 * kernel_gaussian_local_jacobian_t_matvec (src/local_kernels_bindings.cpp:
 * 1358-1427, src/local_kernels.cpp:3155-3262) and f_out
 * kernel_gaussian_local_hessian_matvec (:1246-1356, local_kernels.cpp:2895-3154);
 * with alpha_e both are kernel_gaussian_local_full_matvec (:1429-1530,
 * local_kernels.cpp:3263-3425).  e_out or f_out may be NULL (not
 * computed); f_out needs dx1.  alpha_desc NULL means all-zero force
 * coefficients.  x1, dx1, x2 of element type x_dt, everything else double;
 * q / n host.  FP64 arithmetic (FP64 cuBLAS GEMMs for the pair products). */
kfb_status kfb_local_matvec(const void *x1, const void *dx1, const void *x2,
                            const double *alpha_desc, const double *alpha_e, const int32_t *q1,
                            const int32_t *q2, const int32_t *n1, const int32_t *n2, int nm1,
                            int nm2, int ma1, int ma2, int rep, double sigma, kfb_dtype x_dt,
                            double *e_out, double *f_out, void *stream);

/* ---------------------------------------------------------------------- */
/* FCHL19 descriptors and Jacobians                                        */
/* ---------------------------------------------------------------------- */

/* Descriptor length nelements nRs2 + nelements (nelements + 1) / 2 nRs3 2 nFourier
 * (-1 for invalid sizes).  Replaces fchl19_repr.compute_rep_size
 * (src/fchl19_repr_bindings.cpp:222-230; its nabasis is 2 nFourier). */
int kfb_fchl19_rep_size(int nelements, int nRs2, int nRs3, int nFourier);

/* FCHL19 descriptors of nm padded molecules: coords (nm, ma, 3) device, element
 * indices elem (nm, ma) host int32 in [0, nelements) for the first natoms[m]
 * atoms (host int32, clamped to [0, ma]); rep (nm, ma, rep_size) device and, when
 * grad is not NULL, grad (nm, ma, rep_size, 3 ma) device = d rep[m, i, f] /
 * d coords[m, a, t] at column 3 a + t (the layout of the kernels' dX; padded
 * atoms are zero).  Element type of coords / rep / grad: dt; FP64 arithmetic.
 * Hyper-parameters as fchl19_repr.generate_fchl_acsf (the three-body weight is
 * scaled by sqrt(eta3 / pi) inside, as the reference's binding does); gradients
 * need nFourier = 1.  Replaces fchl19_repr.generate_fchl_acsf /
 * generate_fchl_acsf_and_gradients (src/fchl19_repr_bindings.cpp:52-216,
 * src/fchl19_repr.cpp:89-781) and cuda_fchl19_repr.generate_fchl_acsf /
 * generate_fchl_acsf_and_gradients (src/cuda_fchl19_repr_bindings.cpp:170-290). */
kfb_status kfb_fchl19_repr(const void *coords, const int32_t *elem, const int32_t *natoms,
                           int nm, int ma, int nelements, int nRs2, int nRs3, int nFourier,
                           double eta2, double eta3, double zeta, double rcut, double acut,
                           double two_body_decay, double three_body_decay,
                           double three_body_weight, kfb_dtype dt, void *rep, void *grad,
                           void *stream);

/* ---------------------------------------------------------------------- */
/* Allocation-free entry point                                             */
/* ---------------------------------------------------------------------- */

/* Size of the fixed device scratch array behind kfb_kernel_gaussian_symm_noalloc
 * (held by every GPU that loads the library, until the process exits). */
#define KFB_NOALLOC_SCRATCH_BYTES (64u << 20)

/* The symmetric scalar kernel of kfb_kernel_gaussian_symm with FP64 CUDA-core
 * arithmetic and a double output (layout KFB_DENSE / KFB_RFP_U / KFB_RFP_L),
 * allocating no device memory: for callers that cannot allocate during a call
 * (a host framework that has reserved the device-memory budget up front, or a
 * loop that must not let cudaMalloc / cudaFree synchronise the device).  Its
 * scratch (packed same-label atoms, norms, molecule indices, tile list) lives in
 * one file-scope __device__ array of KFB_NOALLOC_SCRATCH_BYTES; a problem whose
 * scratch exceeds it is rejected with KFB_ERR_INVALID_ARG before any device
 * work (about 11,000 active atoms at rep = 720).  The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) -- make it before
 * any stream capture.  Calls share the array: calls that overlap on the GPU
 * (two streams or two host threads) race.
 * No counterpart in the reference: it is an addition of this library. */
kfb_status kfb_kernel_gaussian_symm_noalloc(const void *x, const int32_t *q, const int32_t *n,
                                            int nm, int ma, int rep, double sigma,
                                            kfb_dtype x_dt, kfb_layout layout, void *out,
                                            void *stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* KFB_H */
