/*
 * kf_oracle.c -- CPU FP64 restatement of the FCHL19 local Gaussian kernel
 * family and the RFP Cholesky KRR solve of andersx/kernelforge.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: it is called by
 * tests/, by __graft_entry__.smoke() and by the cpu_baseline leg of bench.py,
 * and never by the product path (kernelforge_b200/).
 *
 * Every routine is a direct, loop-level statement of the mathematics of the
 * reference routine it cites; no tiling, no BLAS, no OpenMP (except the
 * optional row-parallel pragma, which does not change the summation order of
 * any output entry).  Parity is pinned against the reference itself: see
 * tests/golden/make_golden.py, which builds the reference CPU modules from
 * their sources and records their outputs.
 *
 * Conventions (all arrays C-contiguous, row-major):
 *   X  : (nm, ma, rep)            descriptors
 *   dX : (nm, ma, rep, 3*ma)      descriptor Jacobians dX/dR
 *   Q  : (nm, ma) int32            labels (nuclear charges)
 *   N  : (nm,) int32               active atoms, clamped to [0, ma]
 *   e_ij = exp(-|x_i - x_j|^2 / (2 sigma^2))
 */
#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#define CLAMP_N(v, ma) ((v) < 0 ? 0 : ((v) > (ma) ? (ma) : (v)))

/* ------------------------------------------------------------------------ */
/* RFP index maps (TRANSR='N').                                              */
/* ------------------------------------------------------------------------ */

/* Fortran UPLO='U', 0-based (i <= j).  Same map as rfp_index_upper_N in
 * src/local_kernels.cpp:386-400 (and src/rfp_utils.hpp:14-22). */
size_t kfo_rfp_index_upper(long n, long i, long j) {
    if (i > j) { long t = i; i = j; j = t; }
    const long k = n / 2;
    const long stride = (n % 2 == 0) ? (n + 1) : n;
    if (j >= k) return (size_t)(j - k) * (size_t)stride + (size_t)i;
    return (size_t)i * (size_t)stride + (size_t)(j + k + 1);
}

/* Fortran UPLO='L', 0-based (i >= j).  Same map as rfp_index_lower_N_local in
 * src/cuda_local_kernels.cu:3134-3162 (the GPU modules' packing). */
size_t kfo_rfp_index_lower(long n, long i, long j) {
    if (i < j) { long t = i; i = j; j = t; }
    if (n & 1) {
        const long n1 = (n + 1) / 2;
        if (j < n1) return (size_t)(i + j * n);
        return (size_t)(n + (j - n1) + (i - n1) * n);
    }
    const long nk = n / 2;
    if (j < nk) return (size_t)(1 + i + j * (n + 1));
    return (size_t)((j - nk) + (i - nk) * (n + 1));
}

static size_t rfp_index(long n, long i, long j, int uplo_lower) {
    return uplo_lower ? kfo_rfp_index_lower(n, i, j) : kfo_rfp_index_upper(n, i, j);
}

/* Pack the symmetric dense (n x n) A into RFP.  uplo_lower=0: Fortran 'U'. */
void kfo_full_to_rfp(const double *A, long n, int uplo_lower, double *arf) {
    for (long i = 0; i < n; ++i)
        for (long j = i; j < n; ++j)
            arf[rfp_index(n, i, j, uplo_lower)] = A[i * n + j];
}

/* Unpack RFP into a symmetric dense (n x n) matrix. */
void kfo_rfp_to_full(const double *arf, long n, int uplo_lower, double *A) {
    for (long i = 0; i < n; ++i)
        for (long j = i; j < n; ++j) {
            const double v = arf[rfp_index(n, i, j, uplo_lower)];
            A[i * n + j] = v;
            A[j * n + i] = v;
        }
}

/* ------------------------------------------------------------------------ */
/* Scalar kernels                                                            */
/* ------------------------------------------------------------------------ */

static double sqdist(const double *a, const double *b, int rep) {
    double s = 0.0;
    for (int k = 0; k < rep; ++k) {
        const double d = a[k] - b[k];
        s += d * d;
    }
    return s;
}

/* K[a,b] = sum_{i in a, j in b, q_i == q_j} e_ij.
 * Reference: kernel_gaussian, src/local_kernels.cpp:155-298. */
int kfo_kernel_gaussian(const double *x1, const double *x2, const int *q1, const int *q2,
                        const int *n1, const int *n2, int nm1, int nm2, int ma1, int ma2,
                        int rep, double sigma, double *K) {
    if (!(sigma > 0.0) || !isfinite(sigma)) return 1;
    const double c = -1.0 / (2.0 * sigma * sigma);
#pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < nm1; ++a) {
        const int na = CLAMP_N(n1[a], ma1);
        for (int b = 0; b < nm2; ++b) {
            const int nb = CLAMP_N(n2[b], ma2);
            double kab = 0.0;
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                    if (q1[(size_t)a * ma1 + i] != q2[(size_t)b * ma2 + j]) continue;
                    kab += exp(c * sqdist(&x1[((size_t)a * ma1 + i) * rep],
                                          &x2[((size_t)b * ma2 + j) * rep], rep));
                }
            K[(size_t)a * nm2 + b] = kab;
        }
    }
    return 0;
}

/* Reference: kernel_gaussian_symm, src/local_kernels.cpp:584-758 (both
 * triangles filled). */
int kfo_kernel_gaussian_symm(const double *x, const int *q, const int *n, int nm, int ma,
                             int rep, double sigma, double *K) {
    return kfo_kernel_gaussian(x, x, q, q, n, n, nm, nm, ma, ma, rep, sigma, K);
}

/* Reference: kernel_gaussian_symm_rfp, src/local_kernels.cpp:403-577 (TRANSR='N',
 * UPLO='U'); uplo_lower=1 gives the GPU modules' UPLO='L' packing
 * (src/cuda_local_kernels.cu:3224-3359). */
int kfo_kernel_gaussian_symm_rfp(const double *x, const int *q, const int *n, int nm, int ma,
                                 int rep, double sigma, int uplo_lower, double *arf) {
    double *K = (double *)malloc(sizeof(double) * (size_t)nm * nm);
    if (!K) return 2;
    int rc = kfo_kernel_gaussian_symm(x, q, n, nm, ma, rep, sigma, K);
    if (rc == 0) kfo_full_to_rfp(K, nm, uplo_lower, arf);
    free(K);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Derivative kernels                                                        */
/* ------------------------------------------------------------------------ */

static void offsets(const int *n, int nm, int ma, int *offs, int *total) {
    int s = 0;
    for (int m = 0; m < nm; ++m) {
        offs[m] = s;
        s += 3 * CLAMP_N(n[m], ma);
    }
    *total = s;
}

/* K[a, off2[b] + c] = sum_{i in a, j in b, same label}
 *                     (e_ij / sigma^2) * sum_k dX2[b,j,k,c] (x1[a,i,k] - x2[b,j,k])
 * i.e. +dK/dR2.  Reference: kernel_gaussian_jacobian, src/local_kernels.cpp:791-974. */
int kfo_kernel_gaussian_jacobian(const double *x1, const double *x2, const double *dx2,
                                 const int *q1, const int *q2, const int *n1, const int *n2,
                                 int nm1, int nm2, int ma1, int ma2, int rep, int naq2,
                                 double sigma, double *K) {
    if (!(sigma > 0.0) || !isfinite(sigma)) return 1;
    int *offs2 = (int *)malloc(sizeof(int) * (size_t)(nm2 > 0 ? nm2 : 1));
    int tot2 = 0;
    offsets(n2, nm2, ma2, offs2, &tot2);
    if (tot2 != naq2) { free(offs2); return 1; }
    const double c2 = -1.0 / (2.0 * sigma * sigma), is2 = 1.0 / (sigma * sigma);
    const int ld2 = 3 * ma2;
    memset(K, 0, sizeof(double) * (size_t)nm1 * naq2);
#pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < nm1; ++a) {
        const int na = CLAMP_N(n1[a], ma1);
        double *d = (double *)malloc(sizeof(double) * (size_t)rep);
        for (int b = 0; b < nm2; ++b) {
            const int nb = CLAMP_N(n2[b], ma2);
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                    if (q1[(size_t)a * ma1 + i] != q2[(size_t)b * ma2 + j]) continue;
                    const double *xi = &x1[((size_t)a * ma1 + i) * rep];
                    const double *xj = &x2[((size_t)b * ma2 + j) * rep];
                    double l2 = 0.0;
                    for (int k = 0; k < rep; ++k) { d[k] = xi[k] - xj[k]; l2 += d[k] * d[k]; }
                    const double w = exp(c2 * l2) * is2;
                    const double *J = &dx2[((size_t)b * ma2 + j) * rep * (size_t)ld2];
                    for (int cc = 0; cc < 3 * nb; ++cc) {
                        double s = 0.0;
                        for (int k = 0; k < rep; ++k) s += J[(size_t)k * ld2 + cc] * d[k];
                        K[(size_t)a * naq2 + offs2[b] + cc] += w * s;
                    }
                }
        }
        free(d);
    }
    free(offs2);
    return 0;
}

/* K_t[off1[a] + c, b] = sum (e_ij / sigma^2) * sum_k dX1[a,i,k,c] (x1[a,i,k] - x2[b,j,k])
 * Reference: kernel_gaussian_jacobian_t, src/local_kernels.cpp:991-1166. */
int kfo_kernel_gaussian_jacobian_t(const double *x1, const double *x2, const double *dx1,
                                   const int *q1, const int *q2, const int *n1, const int *n2,
                                   int nm1, int nm2, int ma1, int ma2, int rep, int naq1,
                                   double sigma, double *K) {
    if (!(sigma > 0.0) || !isfinite(sigma)) return 1;
    int *offs1 = (int *)malloc(sizeof(int) * (size_t)(nm1 > 0 ? nm1 : 1));
    int tot1 = 0;
    offsets(n1, nm1, ma1, offs1, &tot1);
    if (tot1 != naq1) { free(offs1); return 1; }
    const double c2 = -1.0 / (2.0 * sigma * sigma), is2 = 1.0 / (sigma * sigma);
    const int ld1 = 3 * ma1;
    memset(K, 0, sizeof(double) * (size_t)naq1 * nm2);
#pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < nm1; ++a) {
        const int na = CLAMP_N(n1[a], ma1);
        double *d = (double *)malloc(sizeof(double) * (size_t)rep);
        for (int b = 0; b < nm2; ++b) {
            const int nb = CLAMP_N(n2[b], ma2);
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                    if (q1[(size_t)a * ma1 + i] != q2[(size_t)b * ma2 + j]) continue;
                    const double *xi = &x1[((size_t)a * ma1 + i) * rep];
                    const double *xj = &x2[((size_t)b * ma2 + j) * rep];
                    double l2 = 0.0;
                    for (int k = 0; k < rep; ++k) { d[k] = xi[k] - xj[k]; l2 += d[k] * d[k]; }
                    const double w = exp(c2 * l2) * is2;
                    const double *J = &dx1[((size_t)a * ma1 + i) * rep * (size_t)ld1];
                    for (int cc = 0; cc < 3 * na; ++cc) {
                        double s = 0.0;
                        for (int k = 0; k < rep; ++k) s += J[(size_t)k * ld1 + cc] * d[k];
                        K[(size_t)(offs1[a] + cc) * nm2 + b] += w * s;
                    }
                }
        }
        free(d);
    }
    free(offs1);
    return 0;
}

/* H[(a,c1),(b,c2)] = sum_{i in a, j in b, same label}
 *     J_i[:,c1]^T [ (e/sigma^2) I - (e/sigma^4) d d^T ] J_j[:,c2],   d = x1_i - x2_j.
 * Output (naq1, naq2) row-major.  Reference: kernel_gaussian_hessian,
 * src/local_kernels.cpp:1171-1419 (static term :1392-1409, rank-1 term
 * :1343-1389, with expd = -e/sigma^4 and expdiag = e/sigma^2 at :1325-1328). */
int kfo_kernel_gaussian_hessian(const double *x1, const double *x2, const double *dx1,
                                const double *dx2, const int *q1, const int *q2, const int *n1,
                                const int *n2, int nm1, int nm2, int ma1, int ma2, int rep,
                                int naq1, int naq2, double sigma, double *H) {
    if (!(sigma > 0.0) || !isfinite(sigma)) return 1;
    int *offs1 = (int *)malloc(sizeof(int) * (size_t)(nm1 > 0 ? nm1 : 1));
    int *offs2 = (int *)malloc(sizeof(int) * (size_t)(nm2 > 0 ? nm2 : 1));
    int tot1 = 0, tot2 = 0;
    offsets(n1, nm1, ma1, offs1, &tot1);
    offsets(n2, nm2, ma2, offs2, &tot2);
    if (tot1 != naq1 || tot2 != naq2) { free(offs1); free(offs2); return 1; }
    const double c2 = -1.0 / (2.0 * sigma * sigma);
    const double is2 = 1.0 / (sigma * sigma), is4 = is2 * is2;
    const int ld1 = 3 * ma1, ld2 = 3 * ma2;
    memset(H, 0, sizeof(double) * (size_t)naq1 * naq2);
#pragma omp parallel for schedule(dynamic)
    for (int a = 0; a < nm1; ++a) {
        const int na = CLAMP_N(n1[a], ma1);
        double *d = (double *)malloc(sizeof(double) * (size_t)rep);
        double *u = (double *)malloc(sizeof(double) * (size_t)(3 * ma1 + 1));
        double *t = (double *)malloc(sizeof(double) * (size_t)(3 * ma2 + 1));
        for (int b = 0; b < nm2; ++b) {
            const int nb = CLAMP_N(n2[b], ma2);
            for (int i = 0; i < na; ++i)
                for (int j = 0; j < nb; ++j) {
                    if (q1[(size_t)a * ma1 + i] != q2[(size_t)b * ma2 + j]) continue;
                    const double *xi = &x1[((size_t)a * ma1 + i) * rep];
                    const double *xj = &x2[((size_t)b * ma2 + j) * rep];
                    double l2 = 0.0;
                    for (int k = 0; k < rep; ++k) { d[k] = xi[k] - xj[k]; l2 += d[k] * d[k]; }
                    const double e = exp(c2 * l2);
                    const double *Ji = &dx1[((size_t)a * ma1 + i) * rep * (size_t)ld1];
                    const double *Jj = &dx2[((size_t)b * ma2 + j) * rep * (size_t)ld2];
                    for (int c = 0; c < 3 * na; ++c) {
                        double s = 0.0;
                        for (int k = 0; k < rep; ++k) s += Ji[(size_t)k * ld1 + c] * d[k];
                        u[c] = s;
                    }
                    for (int c = 0; c < 3 * nb; ++c) {
                        double s = 0.0;
                        for (int k = 0; k < rep; ++k) s += Jj[(size_t)k * ld2 + c] * d[k];
                        t[c] = s;
                    }
                    for (int c1 = 0; c1 < 3 * na; ++c1)
                        for (int cb = 0; cb < 3 * nb; ++cb) {
                            double s = 0.0;
                            for (int k = 0; k < rep; ++k)
                                s += Ji[(size_t)k * ld1 + c1] * Jj[(size_t)k * ld2 + cb];
                            H[(size_t)(offs1[a] + c1) * naq2 + offs2[b] + cb] +=
                                e * is2 * s - e * is4 * u[c1] * t[cb];
                        }
                }
        }
        free(d); free(u); free(t);
    }
    free(offs1); free(offs2);
    return 0;
}

/* Symmetric Hessian; only the lower triangle (row >= col) is filled, the upper
 * triangle stays zero.  Reference: kernel_gaussian_hessian_symm,
 * src/local_kernels.cpp:1421-1655 (lower triangle only, :1498, :1631-1646). */
int kfo_kernel_gaussian_hessian_symm(const double *x, const double *dx, const int *q,
                                     const int *n, int nm, int ma, int rep, int naq,
                                     double sigma, double *H) {
    int rc = kfo_kernel_gaussian_hessian(x, x, dx, dx, q, q, n, n, nm, nm, ma, ma, rep, naq,
                                         naq, sigma, H);
    if (rc) return rc;
    for (long r = 0; r < naq; ++r)
        for (long c = r + 1; c < naq; ++c) H[r * naq + c] = 0.0;
    return 0;
}

/* Reference: kernel_gaussian_hessian_symm_rfp, src/local_kernels.cpp:1664-1900
 * (RFP TRANSR='N', Fortran UPLO='U'). */
int kfo_kernel_gaussian_hessian_symm_rfp(const double *x, const double *dx, const int *q,
                                         const int *n, int nm, int ma, int rep, int naq,
                                         double sigma, int uplo_lower, double *arf) {
    double *H = (double *)malloc(sizeof(double) * (size_t)naq * (naq > 0 ? naq : 1));
    if (!H) return 2;
    int rc = kfo_kernel_gaussian_hessian(x, x, dx, dx, q, q, n, n, nm, nm, ma, ma, rep, naq, naq,
                                         sigma, H);
    if (rc == 0) kfo_full_to_rfp(H, naq, uplo_lower, arf);
    free(H);
    return rc;
}

/* Full energy+force kernel ((nm1+naq1) x (nm2+naq2)).  Blocks:
 *   [0:nm1, 0:nm2]  scalar            [0:nm1, nm2:]  +jacobian(X1, X2, dX2)
 *   [nm1:, 0:nm2]   -jacobian_t(X1, dX1, X2)   [nm1:, nm2:]  hessian
 * Reference: kernel_gaussian_full, src/local_kernels.cpp:1918-2188 (the fe
 * block uses -expdiag, :2058-2072; the ef block +expdiag, :2074-2080). */
int kfo_kernel_gaussian_full(const double *x1, const double *x2, const double *dx1,
                             const double *dx2, const int *q1, const int *q2, const int *n1,
                             const int *n2, int nm1, int nm2, int ma1, int ma2, int rep,
                             int naq1, int naq2, double sigma, double *K) {
    const long R = nm1 + naq1, C = nm2 + naq2;
    double *S = (double *)malloc(sizeof(double) * ((size_t)nm1 * nm2 + 1));
    double *J = (double *)malloc(sizeof(double) * ((size_t)nm1 * naq2 + 1));
    double *Jt = (double *)malloc(sizeof(double) * ((size_t)naq1 * nm2 + 1));
    double *H = (double *)malloc(sizeof(double) * ((size_t)naq1 * naq2 + 1));
    int rc = kfo_kernel_gaussian(x1, x2, q1, q2, n1, n2, nm1, nm2, ma1, ma2, rep, sigma, S);
    if (!rc) rc = kfo_kernel_gaussian_jacobian(x1, x2, dx2, q1, q2, n1, n2, nm1, nm2, ma1, ma2,
                                               rep, naq2, sigma, J);
    if (!rc) rc = kfo_kernel_gaussian_jacobian_t(x1, x2, dx1, q1, q2, n1, n2, nm1, nm2, ma1, ma2,
                                                 rep, naq1, sigma, Jt);
    if (!rc) rc = kfo_kernel_gaussian_hessian(x1, x2, dx1, dx2, q1, q2, n1, n2, nm1, nm2, ma1,
                                              ma2, rep, naq1, naq2, sigma, H);
    if (!rc) {
        for (long r = 0; r < R; ++r)
            for (long c = 0; c < C; ++c) {
                double v;
                if (r < nm1 && c < nm2) v = S[r * nm2 + c];
                else if (r < nm1) v = J[r * naq2 + (c - nm2)];
                else if (c < nm2) v = -Jt[(r - nm1) * nm2 + c];
                else v = H[(r - nm1) * naq2 + (c - nm2)];
                K[r * C + c] = v;
            }
    }
    free(S); free(J); free(Jt); free(H);
    return rc;
}

/* Reference: kernel_gaussian_full_symm, src/local_kernels.cpp:2201-2498 (fully
 * filled symmetric matrix). */
int kfo_kernel_gaussian_full_symm(const double *x, const double *dx, const int *q, const int *n,
                                  int nm, int ma, int rep, int naq, double sigma, double *K) {
    return kfo_kernel_gaussian_full(x, x, dx, dx, q, q, n, n, nm, nm, ma, ma, rep, naq, naq,
                                    sigma, K);
}

/* Reference: kernel_gaussian_full_symm_rfp, src/local_kernels.cpp:2511-2815
 * (RFP TRANSR='N', Fortran UPLO='U' of the BIG = nm+naq matrix). */
int kfo_kernel_gaussian_full_symm_rfp(const double *x, const double *dx, const int *q,
                                      const int *n, int nm, int ma, int rep, int naq,
                                      double sigma, int uplo_lower, double *arf) {
    const long big = nm + naq;
    double *K = (double *)malloc(sizeof(double) * (size_t)big * big);
    if (!K) return 2;
    int rc = kfo_kernel_gaussian_full_symm(x, dx, q, n, nm, ma, rep, naq, sigma, K);
    if (!rc) kfo_full_to_rfp(K, big, uplo_lower, arf);
    free(K);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* Cholesky KRR solve on RFP storage                                         */
/* ------------------------------------------------------------------------ */

/* (K + l2 I) alpha = y with K given in RFP (TRANSR='N').  On exit arf holds the
 * Cholesky factor in the same RFP layout (UPLO='U': K = U^T U; UPLO='L':
 * K = L L^T), as LAPACK dpftrf leaves it.  Returns 0, or the order of the first
 * non-positive leading minor (LAPACK info > 0).
 * Reference: kf::math::solve_cholesky_rfp, src/math.cpp:134-171 (diagonal
 * shift :156-162, dpftrf :165, dpftrs :169). */
int kfo_cho_solve_rfp(double *arf, const double *y, long n, double l2, int uplo_lower,
                      double *alpha) {
    double *A = (double *)malloc(sizeof(double) * (size_t)n * n);
    if (!A) return -1;
    kfo_rfp_to_full(arf, n, uplo_lower, A);
    for (long i = 0; i < n; ++i) A[i * n + i] += l2;
    /* lower Cholesky in place: A = L L^T, L stored in the lower triangle */
    for (long j = 0; j < n; ++j) {
        double s = A[j * n + j];
        for (long k = 0; k < j; ++k) s -= A[j * n + k] * A[j * n + k];
        if (!(s > 0.0)) { free(A); return (int)(j + 1); }
        const double ljj = sqrt(s);
        A[j * n + j] = ljj;
        for (long i = j + 1; i < n; ++i) {
            double t = A[i * n + j];
            for (long k = 0; k < j; ++k) t -= A[i * n + k] * A[j * n + k];
            A[i * n + j] = t / ljj;
        }
    }
    /* forward: L z = y ; backward: L^T alpha = z */
    for (long i = 0; i < n; ++i) {
        double t = y[i];
        for (long k = 0; k < i; ++k) t -= A[i * n + k] * alpha[k];
        alpha[i] = t / A[i * n + i];
    }
    for (long i = n - 1; i >= 0; --i) {
        double t = alpha[i];
        for (long k = i + 1; k < n; ++k) t -= A[k * n + i] * alpha[k];
        alpha[i] = t / A[i * n + i];
    }
    /* store the factor back: U = L^T for 'U', L for 'L' */
    for (long i = 0; i < n; ++i)
        for (long j = i; j < n; ++j)
            arf[rfp_index(n, i, j, uplo_lower)] = A[j * n + i];
    free(A);
    return 0;
}
