// FCHL19 atomic descriptors and their Jacobians dX/dR on the GPU (the
// upstream producer of the kernels' X and dX: src/fchl19_repr.cpp:89-306
// forward, :308-781 values + gradients; src/cuda_fchl19_repr.cu).
//
// Descriptor of centre atom i (rep = nelem nRs2 + npair nRs3 nab, npair =
// nelem (nelem + 1) / 2, nab = 2 nFourier):
//   two-body, channel elem_j nRs2 + k, over neighbours j with r_ij <= rcut:
//     g_k(r) = decay2(r) / (sig sqrt(2 pi) r^p2) exp(-(log Rs2_k - mu)^2 / (2 sig^2)) / Rs2_k,
//     sig^2 = log(1 + eta2 / r^2), mu = log r - sig^2 / 2, decay(r) = (cos(pi r / cut) + 1) / 2
//   three-body, channel pair(elem_j, elem_k) nRs3 nab + l nab + a, over j < k
//   with r_ij, r_ik <= acut:
//     atm   = w3 (1 + 3 cos_i cos_j cos_k) / (r_ij r_ik r_jk)^p3,  w3 = sqrt(eta3 / pi) w
//     rad_l = exp(-eta3 ((r_ij + r_ik) / 2 - Rs3_l)^2) decay3(r_ij) decay3(r_ik)
//     ang   = 2 exp(-(zeta o)^2 / 2) [cos(o theta_i), sin(o theta_i)],  o = 1, 3, 5, ...
// Rs2_k = rcut (k + 1) / nRs2, Rs3_l = acut (l + 1) / nRs3.
//
// GPU layout: block per (molecule, centre i); each warp owns partner atoms o
// and computes every column of dX[i, :, 3o .. 3o+2] itself (two-body from the
// pair (i, o), three-body from the triples (i; o, q)): no atomics on dX.  The
// centre's own columns follow from translation invariance of every term,
//   dX[i, :, 3i + t] = -sum_{o != i} dX[i, :, 3o + t],
// summed in shared memory.  In the three-body loop the lanes first build the
// geometry of 32 triples (one partner each) into shared slots, then lane l
// takes radial channel l over the stored triples, with its accumulators per
// partner element in registers.  Values of
// the descriptor are summed in shared memory (each triple once, by its owner
// o < q).  Arithmetic in FP64; outputs FP64 or FP32.
#include <cmath>
#include <vector>

#include "kfb_internal.h"

namespace kfb {

namespace {

constexpr int REPR_MAX_ELEM = 8;    // element channels held in registers per lane
constexpr int REPR_WARPS = 8;
constexpr double REPR_EPS = 1e-12;

struct ReprParams {
    int nelem, nRs2, nRs3, nab;
    int rep, three_off;
    double eta2, eta3, rcut, acut, p2, p3, w3;
    double ang_w[8];  // 2 exp(-(zeta o)^2 / 2) for o = 1, 3, ..., 2 nab/2 - 1
};

__host__ __device__ inline int pair_channel(int nelem, int p, int q) {
    if (p > q) {
        const int t = p;
        p = q;
        q = t;
    }
    return p * nelem - p * (p + 1) / 2 + q;
}

__device__ inline double half_cos_decay(double r, double cut) {
    return 0.5 * (cos(M_PI * r / cut) + 1.0);
}

// Two-body radial value and d/dr for basis function k.
__device__ inline void two_body(const ReprParams &P, double r, int k, double &v, double &dv) {
    const double t = P.eta2 / fmax(r * r, REPR_EPS);
    const double s2 = log1p(t);
    const double sig = sqrt(fmax(s2, 0.0));
    v = dv = 0.0;
    if (sig < REPR_EPS) return;
    const double mu = log(r) - 0.5 * s2;
    const double ds2 = -2.0 * t / (r * (1.0 + t));
    const double dsig = ds2 / (2.0 * sig);
    const double dmu = 1.0 / r - 0.5 * ds2;
    const double dec = half_cos_decay(r, P.rcut);
    const double ddec = -0.5 * M_PI / P.rcut * sin(M_PI * r / P.rcut);
    const double rp = pow(r, -P.p2);
    const double c = 1.0 / (sqrt(2.0 * M_PI) * sig);
    const double pref = dec * rp * c;
    const double dpref = (ddec * rp - dec * P.p2 * rp / r) * c - pref * dsig / sig;
    const double Rs = P.rcut * (k + 1) / P.nRs2;
    const double L = log(Rs) - mu;
    const double g = exp(-0.5 * L * L / s2);
    const double dg = g * (L * dmu / s2 + 0.5 * L * L * ds2 / (s2 * s2));
    v = pref * g / Rs;
    dv = (dpref * g + pref * dg) / Rs;
}

// Angular basis of the centre angle: cos(o theta), sin(o theta) times the
// harmonic weights, o = 1, 3, ... (Chebyshev recurrence on cos theta).
__device__ inline void angular_basis(const ReprParams &P, double c, double s, double *ang) {
    ang[0] = P.ang_w[0] * c;
    ang[1] = P.ang_w[0] * s;
    if (P.nab <= 2) return;
    double cm2 = 1.0, sm2 = 0.0, cm1 = c, sm1 = s;
    int h = 1;
    for (int n = 2; h < P.nab / 2; ++n) {
        const double cn = 2.0 * c * cm1 - cm2, sn = 2.0 * c * sm1 - sm2;
        cm2 = cm1;
        sm2 = sm1;
        cm1 = cn;
        sm1 = sn;
        if (n == 2 * h + 1) {
            ang[2 * h] = P.ang_w[h] * cn;
            ang[2 * h + 1] = P.ang_w[h] * sn;
            ++h;
        }
    }
}

struct Vec3 {
    double x, y, z;
};
__device__ inline Vec3 sub(const Vec3 &a, const Vec3 &b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ inline double dot(const Vec3 &a, const Vec3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ inline Vec3 axpby(double a, const Vec3 &u, double b, const Vec3 &v) {
    return {a * u.x + b * v.x, a * u.y + b * v.y, a * u.z + b * v.z};
}

// The triple (i; o, q) seen from its owner o: the angle terms and the
// gradients with respect to R_o of atm, cos_i and the radial/decay factors.
struct Triple {
    double cos_i, sin_i;   // angle at the centre (cos clamped to [-1, 1])
    double atm;            // w3 (1 + 3 cos_i cos_o cos_q) / (r_io r_iq r_oq)^p3
    double dec;            // decay3(r_io) decay3(r_iq)
    double rbar;           // (r_io + r_iq) / 2
    Vec3 datm;             // d atm / dR_o
    Vec3 dcos;             // d cos_i / dR_o, times (r_io r_iq) / sqrt(max(1e-10, (r_io r_iq)^2 - dot^2))
    Vec3 ddec;             // d dec / dR_o
    Vec3 eio;              // (R_o - R_i) / r_io
};

__device__ inline Triple make_triple(const ReprParams &P, const Vec3 &Ri, const Vec3 &Ro,
                                     const Vec3 &Rq, double r_io, double r_iq) {
    Triple T;
    const Vec3 dio = sub(Ro, Ri), diq = sub(Rq, Ri), doq = sub(Rq, Ro);
    const double r_oq = sqrt(dot(doq, doq));
    const Vec3 eio = axpby(1.0 / r_io, dio, 0.0, dio);
    const Vec3 eiq = axpby(1.0 / r_iq, diq, 0.0, diq);
    const Vec3 eoq = axpby(1.0 / r_oq, doq, 0.0, doq);
    const double ci_raw = dot(eio, eiq);
    const double ci = fmin(1.0, fmax(-1.0, ci_raw));
    const double co = -dot(eio, eoq);  // angle at o: (R_i - R_o) . (R_q - R_o)
    const double cq = dot(eiq, eoq);   // angle at q: (R_i - R_q) . (R_o - R_q)
    T.cos_i = ci;
    T.sin_i = sqrt(fmax(0.0, 1.0 - ci * ci));
    const double prod = r_io * r_iq * r_oq;
    const double inv_p = pow(prod, -P.p3);
    T.atm = P.w3 * (1.0 + 3.0 * ci * co * cq) * inv_p;
    // d cos / dR_o of the three angles
    const Vec3 dci = axpby(1.0 / r_io, eiq, -ci_raw / r_io, eio);
    const Vec3 u = axpby(-1.0, eio, 0.0, eio);  // (R_i - R_o) / r_io
    const Vec3 dco = axpby(-1.0 / r_io, axpby(1.0, eoq, -co, u), -1.0 / r_oq, axpby(1.0, u, -co, eoq));
    const Vec3 a = axpby(-1.0, eiq, 0.0, eiq);  // (R_i - R_q) / r_iq
    const Vec3 b = axpby(-1.0, eoq, 0.0, eoq);  // (R_o - R_q) / r_oq
    const Vec3 dcq = axpby(1.0 / r_oq, a, -cq / r_oq, b);
    const Vec3 dlogp = axpby(1.0 / r_io, eio, -1.0 / r_oq, eoq);
    Vec3 d = axpby(co * cq, dci, ci * cq, dco);
    d = axpby(1.0, d, ci * co, dcq);
    T.datm = axpby(3.0 * P.w3 * inv_p, d, -P.p3 * T.atm, dlogp);
    // angle derivative scaled as the reference does near collinear triples
    const double dt = dot(dio, diq);
    const double den = sqrt(fmax(1e-10, r_io * r_io * r_iq * r_iq - dt * dt));
    T.dcos = axpby(r_io * r_iq / den, dci, 0.0, dci);
    const double dio_dec = half_cos_decay(r_io, P.acut), diq_dec = half_cos_decay(r_iq, P.acut);
    T.dec = dio_dec * diq_dec;
    T.ddec = axpby(-0.5 * M_PI / P.acut * sin(M_PI * r_io / P.acut) * diq_dec, eio, 0.0, eio);
    T.rbar = 0.5 * (r_io + r_iq);
    T.eio = eio;
    return T;
}

struct TripleSlot {
    Triple T;
    int q, eq;  // partner atom (-1: empty slot) and its element
};

template <class TO, bool GRAD>
__global__ void __launch_bounds__(REPR_WARPS * 32) fchl19_kernel(
    const TO *__restrict__ coords, const int *__restrict__ elem, const int *__restrict__ natoms,
    int ma, ReprParams P, TO *__restrict__ rep_out, TO *__restrict__ grad_out) {
    extern __shared__ __align__(16) unsigned char rp_raw[];
    double *R = reinterpret_cast<double *>(rp_raw);  // [ma][3]
    double *xs = R + 3 * ma;                         // [rep] values of centre i
    double *gc = xs + P.rep;                         // [rep][3] centre columns (GRAD)
    TripleSlot *tslots = reinterpret_cast<TripleSlot *>(gc + (GRAD ? 3 * P.rep : 0));  // [warps][32]
    int *el = reinterpret_cast<int *>(tslots + REPR_WARPS * 32);                         // [ma]
    const int m = blockIdx.y, i = blockIdx.x;
    const int n = min(max(natoms[m], 0), ma);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rep = P.rep, ld = 3 * ma;
    TO *xo = rep_out + ((size_t)m * ma + i) * rep;
    TO *go = GRAD ? grad_out + ((size_t)m * ma + i) * rep * (size_t)ld : nullptr;
    if (i >= n) {  // padded centre: zeros
        for (int e = threadIdx.x; e < rep; e += blockDim.x) xo[e] = TO(0);
        if (GRAD)
            for (size_t e = threadIdx.x; e < (size_t)rep * ld; e += blockDim.x) go[e] = TO(0);
        return;
    }
    for (int e = threadIdx.x; e < 3 * n; e += blockDim.x) R[e] = (double)coords[(size_t)m * ma * 3 + e];
    for (int e = threadIdx.x; e < n; e += blockDim.x) el[e] = elem[(size_t)m * ma + e];
    for (int e = threadIdx.x; e < rep; e += blockDim.x) xs[e] = 0.0;
    if (GRAD)
        for (int e = threadIdx.x; e < 3 * rep; e += blockDim.x) gc[e] = 0.0;
    __syncthreads();
    const Vec3 Ri{R[3 * i], R[3 * i + 1], R[3 * i + 2]};
    const int npair_rows = P.nRs3 * P.nab;
    for (int o = warp; o < ma; o += REPR_WARPS) {
        if (o >= n || o == i) {
            // columns of padded atoms are zero; the centre's are written below
            if (GRAD && o >= n)
                for (int e = lane; e < 3 * rep; e += 32)
                    go[(size_t)(e / 3) * ld + 3 * o + e % 3] = TO(0);
            continue;
        }
        const Vec3 Ro{R[3 * o], R[3 * o + 1], R[3 * o + 2]};
        const Vec3 dio = sub(Ro, Ri);
        const double r_io = sqrt(dot(dio, dio));
        const int eo = el[o];
        // ---- two-body: pair (i, o), channel eo nRs2 + k
        if (GRAD) {
            // every two-body column of owner o: zero except the channel block of eo
            for (int e = lane; e < P.three_off; e += 32) {
                const int k = e - eo * P.nRs2;
                double v = 0.0, dv = 0.0;
                if (k >= 0 && k < P.nRs2 && r_io <= P.rcut) two_body(P, r_io, k, v, dv);
                const double g[3] = {dv * dio.x / r_io, dv * dio.y / r_io, dv * dio.z / r_io};
#pragma unroll
                for (int t = 0; t < 3; ++t) {
                    go[(size_t)e * ld + 3 * o + t] = (TO)g[t];
                    if (g[t] != 0.0) atomicAdd(&gc[3 * e + t], -g[t]);
                }
                if (v != 0.0) atomicAdd(&xs[e], v);
            }
        } else if (r_io <= P.rcut) {
            for (int k = lane; k < P.nRs2; k += 32) {
                double v, dv;
                two_body(P, r_io, k, v, dv);
                if (v != 0.0) atomicAdd(&xs[eo * P.nRs2 + k], v);
            }
        }
        // ---- three-body: triples (i; o, q).  Lanes first build the geometry of
        // up to 32 partners q (one triple each) into the warp's shared slots,
        // then lane l takes radial channel l over every stored triple.
        const bool o_in = r_io <= P.acut;
        TripleSlot *slots = tslots + (size_t)warp * 32;
        for (int l0 = 0; l0 < P.nRs3; l0 += 32) {
            const int l = l0 + lane;
            const bool lv = l < P.nRs3;
            const double Rs3 = P.acut * (l + 1) / P.nRs3;
            double acc[REPR_MAX_ELEM][2][3];
#pragma unroll
            for (int e = 0; e < REPR_MAX_ELEM; ++e)
#pragma unroll
                for (int a = 0; a < 2; ++a)
#pragma unroll
                    for (int t = 0; t < 3; ++t) acc[e][a][t] = 0.0;
            for (int q0 = 0; o_in && q0 < n; q0 += 32) {
                {
                    const int q = q0 + lane;
                    TripleSlot &S = slots[lane];
                    S.q = -1;
                    if (q < n && q != i && q != o) {
                        const Vec3 Rq{R[3 * q], R[3 * q + 1], R[3 * q + 2]};
                        const Vec3 diq = sub(Rq, Ri);
                        const double r_iq = sqrt(dot(diq, diq));
                        if (r_iq <= P.acut) {
                            S.T = make_triple(P, Ri, Ro, Rq, r_io, r_iq);
                            S.q = q;
                            S.eq = el[q];
                        }
                    }
                }
                __syncwarp();
                const int qn = min(32, n - q0);
                for (int sI = 0; sI < qn; ++sI) {
                    const int q = slots[sI].q;
                    if (q < 0) continue;  // warp-uniform
                    const Triple &T = slots[sI].T;
                    const int eq = slots[sI].eq;
                    const double dr = T.rbar - Rs3;
                    const double rad = exp(-P.eta3 * dr * dr);
                    double ang[16];
                    angular_basis(P, T.cos_i, T.sin_i, ang);
                    const int ch = P.three_off + pair_channel(P.nelem, eo, eq) * npair_rows;
                    if (lv && o < q)
                        for (int a = 0; a < P.nab; ++a)
                            atomicAdd(&xs[ch + l * P.nab + a], ang[a] * rad * T.atm * T.dec);
                    if (GRAD && lv) {
                        // d V / dR_o, V = ang_a rad atm dec (o = 1 harmonic pair)
                        const double drad = -P.eta3 * dr * rad;  // d rad / d r_io
                        const double wv = P.ang_w[0];
                        const double dang[2] = {wv * T.sin_i, -wv * T.cos_i};
#pragma unroll
                        for (int a = 0; a < 2; ++a) {
                            const double base = rad * T.dec;
                            const Vec3 g = axpby(
                                1.0,
                                axpby(ang[a] * base, T.datm, dang[a] * base * T.atm, T.dcos),
                                1.0,
                                axpby(ang[a] * T.atm * drad * T.dec, T.eio,
                                      ang[a] * T.atm * rad, T.ddec));
#pragma unroll
                            for (int e = 0; e < REPR_MAX_ELEM; ++e) {
                                if (e == eq) {
                                    acc[e][a][0] += g.x;
                                    acc[e][a][1] += g.y;
                                    acc[e][a][2] += g.z;
                                }
                            }
                        }
                    }
                }
                __syncwarp();  // slots read by every lane before the next fill
            }
            if (GRAD) {
                // write owner o's three-body columns for channel l (every pair block)
                for (int pe = 0; pe < P.nelem * (P.nelem + 1) / 2; ++pe) {
                    // pair block pe involves eo?  then its partner element is the other one
                    int partner = -1;
                    for (int e = 0; e < P.nelem && e < REPR_MAX_ELEM; ++e)
                        if (pair_channel(P.nelem, eo, e) == pe) partner = e;
                    if (!lv) continue;
#pragma unroll
                    for (int a = 0; a < 2; ++a) {  // nab == 2 with gradients
                        const int ch = P.three_off + pe * npair_rows + l * P.nab + a;
                        double g[3] = {0.0, 0.0, 0.0};
                        if (partner >= 0) {
#pragma unroll
                            for (int e = 0; e < REPR_MAX_ELEM; ++e)
                                if (e == partner)
#pragma unroll
                                    for (int t = 0; t < 3; ++t) g[t] = acc[e][a][t];
                        }
#pragma unroll
                        for (int t = 0; t < 3; ++t) {
                            go[(size_t)ch * ld + 3 * o + t] = (TO)g[t];
                            if (g[t] != 0.0) atomicAdd(&gc[3 * ch + t], -g[t]);
                        }
                    }
                }
            }
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < rep; e += blockDim.x) xo[e] = (TO)xs[e];
    if (GRAD)
        for (int e = threadIdx.x; e < 3 * rep; e += blockDim.x)
            go[(size_t)(e / 3) * ld + 3 * i + e % 3] = (TO)gc[e];
}

}  // namespace

}  // namespace kfb

using namespace kfb;

extern "C" {

int kfb_fchl19_rep_size(int nelements, int nRs2, int nRs3, int nFourier) {
    if (nelements <= 0 || nRs2 < 0 || nRs3 < 0 || nFourier <= 0) return -1;
    return nelements * nRs2 + nelements * (nelements + 1) / 2 * nRs3 * 2 * nFourier;
}

kfb_status kfb_fchl19_repr(const void *coords, const int32_t *elem, const int32_t *natoms,
                           int nm, int ma, int nelements, int nRs2, int nRs3, int nFourier,
                           double eta2, double eta3, double zeta, double rcut, double acut,
                           double two_body_decay, double three_body_decay,
                           double three_body_weight, kfb_dtype dt, void *rep, void *grad,
                           void *stream) {
    if (!coords || !elem || !natoms || !rep) return set_error(KFB_ERR_INVALID_ARG, "null pointer");
    if (nm < 0 || ma <= 0) return set_error(KFB_ERR_INVALID_ARG, "nm >= 0 and max_atoms > 0 required");
    for (int m = 0; m < nm; ++m) {
        const int n = natoms[m] < 0 ? 0 : (natoms[m] > ma ? ma : natoms[m]);
        for (int i = 0; i < n; ++i) {
            const int e = elem[(size_t)m * ma + i];
            if (e < 0 || e >= nelements)
                return set_error(KFB_ERR_INVALID_ARG,
                                 "element index %d of atom %d in molecule %d outside [0, %d)", e,
                                 i, m, nelements);
        }
    }
    if (nelements <= 0 || nelements > REPR_MAX_ELEM)
        return set_error(KFB_ERR_INVALID_ARG, "nelements must be in [1, %d]", REPR_MAX_ELEM);
    if (nRs2 <= 0 || nRs3 <= 0 || nFourier <= 0 || nFourier > 8)
        return set_error(KFB_ERR_INVALID_ARG, "nRs2, nRs3 > 0 and nFourier in [1, 8] required");
    if (grad && nFourier != 1)
        return set_error(KFB_ERR_INVALID_ARG, "gradients are defined for nFourier = 1");
    if (!(rcut > 0) || !(acut > 0) || !(eta2 > 0) || !(eta3 > 0))
        return set_error(KFB_ERR_INVALID_ARG, "rcut, acut, eta2, eta3 must be > 0");
    if (nm == 0) return KFB_OK;
    ReprParams P{};
    P.nelem = nelements;
    P.nRs2 = nRs2;
    P.nRs3 = nRs3;
    P.nab = 2 * nFourier;
    P.three_off = nelements * nRs2;
    P.rep = kfb_fchl19_rep_size(nelements, nRs2, nRs3, nFourier);
    P.eta2 = eta2;
    P.eta3 = eta3;
    P.rcut = rcut;
    P.acut = acut;
    P.p2 = two_body_decay;
    P.p3 = three_body_decay;
    P.w3 = std::sqrt(eta3 / M_PI) * three_body_weight;
    for (int h = 0; h < nFourier; ++h) {
        const double t = zeta * (2 * h + 1);
        P.ang_w[h] = 2.0 * std::exp(-0.5 * t * t);
    }
    const bool g = grad != nullptr;
    const size_t smem = (size_t)(3 * ma + P.rep + (g ? 3 * P.rep : 0)) * sizeof(double) +
                        (size_t)REPR_WARPS * 32 * sizeof(TripleSlot) + (size_t)ma * sizeof(int);
    if (smem > 200 * 1024)
        return set_error(KFB_ERR_INVALID_ARG, "descriptor too large for one block (%zu bytes)", smem);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::vector<int> ev(elem, elem + (size_t)nm * ma), nv(natoms, natoms + nm);
    DevBuf d_elem, d_n;
    KFB_TRY(upload(d_elem, ev, s));
    KFB_TRY(upload(d_n, nv, s));
    const int *de = d_elem.as<int>(), *dn = d_n.as<int>();
    const dim3 grid((unsigned)ma, (unsigned)nm);
    auto launch = [&](auto kern) -> kfb_status {
        if (smem > 48 * 1024)
            KFB_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)smem));
        return KFB_OK;
    };
    if (dt == KFB_F64) {
        if (g) {
            KFB_TRY(launch(fchl19_kernel<double, true>));
            fchl19_kernel<double, true><<<grid, REPR_WARPS * 32, smem, s>>>(
                static_cast<const double *>(coords), de, dn, ma, P,
                static_cast<double *>(rep), static_cast<double *>(grad));
        } else {
            KFB_TRY(launch(fchl19_kernel<double, false>));
            fchl19_kernel<double, false><<<grid, REPR_WARPS * 32, smem, s>>>(
                static_cast<const double *>(coords), de, dn, ma, P,
                static_cast<double *>(rep), nullptr);
        }
    } else {
        if (g) {
            KFB_TRY(launch(fchl19_kernel<float, true>));
            fchl19_kernel<float, true><<<grid, REPR_WARPS * 32, smem, s>>>(
                static_cast<const float *>(coords), de, dn, ma, P,
                static_cast<float *>(rep), static_cast<float *>(grad));
        } else {
            KFB_TRY(launch(fchl19_kernel<float, false>));
            fchl19_kernel<float, false><<<grid, REPR_WARPS * 32, smem, s>>>(
                static_cast<const float *>(coords), de, dn, ma, P,
                static_cast<float *>(rep), nullptr);
        }
    }
    KFB_CUDA_TRY(cudaGetLastError());
    return KFB_OK;
}

}  // extern "C"
