/*
 * sc_oracle.c -- CPU restatement of OPAL's space-charge tracking step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA product
 * path and the timed CPU baseline; nothing in the product links or calls it.
 * It restates, in plain sequential FP64 C, the algorithms of the OPAL 2.x
 * reference (paths below are relative to the reference source tree):
 *
 *   half drift           src/Steppers/BorisPusher.h:116-124,
 *                        src/Classic/Algorithms/PartBunchBase.hpp:468-513,
 *                        src/Algorithms/ParallelTTracker.h:448-455
 *   Boris kick           src/Steppers/BorisPusher.h:56-113, ParallelTTracker.h:442-446
 *   beam parameters      src/Classic/Algorithms/PartBunchBase.hpp:1178-1219 (bounds),
 *                        :1529-1614 (calcBeamParameters), :2185-2259 (calcMoments)
 *   mesh per step        PartBunchBase.hpp:802-884 (boundp), PartBunch.cpp:1109-1120
 *   CIC scatter/gather   ippl/src/Particle/IntCIC.h:818-858, :935-975,
 *                        ippl/src/Meshes/UniformCartesian.hpp:1025-1039, :1084-1097
 *   self fields          src/Classic/Algorithms/PartBunch.cpp:482-647
 *   Poisson solve        src/Solvers/FFTPoissonSolver.cpp:337-382 (computePotential),
 *                        :459-522 (integratedGreensFunction), :641-664 (mirrorRhoField)
 *   3-D RC FFT           ippl/src/FFT/FFT.hpp:709-740 (normalisation), :1078-1340, :1483-1710,
 *                        ippl/src/FFT/fftpack_FFT.h:194-245 (half-complex repack)
 *   gradient             ippl/src/Meshes/UniformCartesian.hpp:2129-2203
 *   frames               src/Classic/Algorithms/Quaternion.cpp:34-150,
 *                        src/Classic/Algorithms/CoordinateSystemTrafo.{h:77-85,cpp}
 *   step loop            src/Algorithms/ParallelTTracker.cpp:343-388, :546-592, :1123-1212
 *   constants            src/Classic/Physics/Physics.h:31-76, src/Track/TrackRun.cpp:423,
 *                        src/Structure/Beam.cpp:64,260-263
 *
 * Floating-point expressions keep the reference's operand order so that the
 * restatement rounds like the reference wherever the order is defined.
 * Build with -ffp-contract=off (no fused multiply-add contraction).
 *
 * The 1-D FFT engine is pluggable: by default a project-written mixed-radix
 * FFT with FFTPACK's conventions; tests switch in the reference's own
 * ippl/src/FFT/fftpack.cpp (compiled from source into oracle/_ref/) through
 * sco_set_fft_engine().
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "sc_oracle.h"

#ifdef _OPENMP
#include <omp.h>
#include <quadmath.h>
#endif

/* ------------------------------------------------------------------------ */
/* constants: Physics.h:31,52,58,70,76; Beam.cpp:64; TrackRun.cpp:423        */
/* ------------------------------------------------------------------------ */
#define SCO_PI 3.14159265358979323846
#define SCO_C 299792458.0
#define SCO_EPS0 8.854187817e-12

/* Host threads for the timed multi-core baseline (1 = the sequential
 * restatement).  With more threads, particle loops, FFT strips and the
 * Green's function run in parallel; the deposit goes to per-thread grids
 * merged in thread order and sums are combined in thread order, so a run is
 * reproducible for a fixed thread count. */
static int g_threads = 1;

/* Exact mode (off by default, i.e. the reference's own arithmetic):
 *  - the Green's function's atan / log correctly rounded (quad precision);
 *  - the particle sums (moments, the mean momentum behind gamma_z and the
 *    beam frame, the sum of gamma) order-independent: every term v becomes
 *    the integer trunc(v 2^72) (|v| < 2^55), the integers are added exactly
 *    in 128 bits and the total is rounded to a double once.
 * The reference sums particles in storage order on each rank and then across
 * ranks (MPI_Allreduce), so its last bits depend on the rank count; through
 * gamma_z and the eight-corner cancellation of the Green's function one ulp
 * of such a sum moves the field by ~1e-11.  The exact mode fixes one answer. */
static int g_exact = 0;
void sco_set_exact(int on) { g_exact = on != 0; }
int sco_get_exact(void) { return g_exact; }

typedef __int128 sco_i128;
#define SCO_EX_FRAC 72
static sco_i128 ex_from(double v) {
    uint64_t bits;
    memcpy(&bits, &v, sizeof bits);
    const int e = (int)((bits >> 52) & 0x7ff);
    if (e == 0) return 0; /* zero or subnormal */
    const uint64_t m = (bits & 0xfffffffffffffull) | (1ull << 52);
    const int sh = e - 1075 + SCO_EX_FRAC;
    unsigned __int128 mag;
    if (sh >= 0)
        mag = sh < 75 ? ((unsigned __int128)m << sh) : ((unsigned __int128)m << 74);
    else
        mag = sh > -53 ? (unsigned __int128)(m >> (-sh)) : 0;
    return (bits >> 63) ? -(sco_i128)mag : (sco_i128)mag;
}
/* (double) of a 128-bit integer rounds to nearest-even; the scaling is exact */
static double ex_to_double(sco_i128 x) { return ldexp((double)x, -SCO_EX_FRAC); }
#define SCO_PAR _Pragma("omp parallel for num_threads(g_threads) if(g_threads > 1) schedule(static)")
void sco_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int sco_get_threads(void) { return g_threads; }
int sco_max_threads(void) {
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

double sco_const_c(void) { return SCO_C; }
double sco_const_electron_mass_ev(void) { return 0.51099892e-03 * 1.0e9; }
double sco_const_coupling(void) { return 1.0 / (4 * SCO_PI * SCO_EPS0); }

/* ------------------------------------------------------------------------ */
/* small vector algebra with IPPL's evaluation order                        */
/* (TSVMetaDot.h:62-69, :255-264; TSVMetaCross.h:38-49)                     */
/* ------------------------------------------------------------------------ */
static inline double dot3(const double* a, const double* b) {
    return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}
static inline void cross3(const double* a, const double* b, double* r) {
    double r0 = a[1] * b[2] - a[2] * b[1];
    double r1 = a[2] * b[0] - a[0] * b[2];
    double r2 = a[0] * b[1] - a[1] * b[0];
    r[0] = r0; r[1] = r1; r[2] = r2;
}
/* Tenzor (row-major, Tenzor.h:202-210) dot Vektor */
static inline void matvec(const double* M, const double* v, double* r) {
    double r0 = M[0] * v[0] + M[1] * v[1] + M[2] * v[2];
    double r1 = M[3] * v[0] + M[4] * v[1] + M[5] * v[2];
    double r2 = M[6] * v[0] + M[7] * v[1] + M[8] * v[2];
    r[0] = r0; r[1] = r1; r[2] = r2;
}

/* ------------------------------------------------------------------------ */
/* quaternions and coordinate-system transformations                        */
/* ------------------------------------------------------------------------ */
/* Quaternion::operator*= (Quaternion.cpp:85-93) */
static void quat_mul(const double* a, const double* b, double* r) {
    double ai[3] = {a[1], a[2], a[3]}, bi[3] = {b[1], b[2], b[3]}, c[3];
    cross3(ai, bi, c);
    double r0 = a[0] * b[0] - dot3(ai, bi);
    double r1 = a[0] * bi[0] + b[0] * ai[0] + c[0];
    double r2 = a[0] * bi[1] + b[0] * ai[1] + c[1];
    double r3 = a[0] * bi[2] + b[0] * ai[2] + c[2];
    r[0] = r0; r[1] = r1; r[2] = r2; r[3] = r3;
}
static double quat_norm(const double* q) { /* Quaternion.h:74-77: dot of the 4-vector */
    return q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
}
static void quat_normalize(double* q) { /* Quaternion.cpp:102-112 */
    double len = sqrt(quat_norm(q));
    q[0] /= len; q[1] /= len; q[2] /= len; q[3] /= len;
}
/* Quaternion::rotate (Quaternion.cpp:122-132): (q * (v * q^*)).imag */
static void quat_rotate(const double* q, const double* v, double* r) {
    double qv[4] = {0.0, v[0], v[1], v[2]};
    double qc[4] = {q[0], -q[1], -q[2], -q[3]};
    double t[4], u[4];
    quat_mul(qv, qc, t);
    quat_mul(q, t, u);
    r[0] = u[1]; r[1] = u[2]; r[2] = u[3];
}
/* Quaternion::getRotationMatrix (Quaternion.cpp:134-149), row-major */
static void quat_rotmat(const double* qin, double* M) {
    double q[4] = {qin[0], qin[1], qin[2], qin[3]};
    quat_normalize(q);
    M[0] = 1 - 2 * (q[2] * q[2] + q[3] * q[3]);
    M[1] = 2 * (-q[0] * q[3] + q[1] * q[2]);
    M[2] = 2 * (q[0] * q[2] + q[1] * q[3]);
    M[3] = 2 * (q[0] * q[3] + q[1] * q[2]);
    M[4] = 1 - 2 * (q[1] * q[1] + q[3] * q[3]);
    M[5] = 2 * (-q[0] * q[1] + q[2] * q[3]);
    M[6] = 2 * (-q[0] * q[2] + q[1] * q[3]);
    M[7] = 2 * (q[0] * q[1] + q[2] * q[3]);
    M[8] = 1 - 2 * (q[1] * q[1] + q[2] * q[2]);
}

/* getQuaternion(u, ref) (Quaternion.cpp:34-68).  Returns 0, or -1 when u is
 * anti-parallel to ref (the reference then draws a random axis; this
 * restatement refuses that case) or when |u| < 1e-12. */
int sco_get_quaternion(const double* uin, const double* refin, double* q) {
    const double tol = 1e-12;
    double u[3] = {uin[0], uin[1], uin[2]}, ref[3] = {refin[0], refin[1], refin[2]};
    double lu = sqrt(dot3(u, u)), lr = sqrt(dot3(ref, ref));
    if (lu < 1e-12 || lr < 1e-12) return -1;
    u[0] /= lu; u[1] /= lu; u[2] /= lu;
    ref[0] /= lr; ref[1] /= lr; ref[2] /= lr;
    double axis[3];
    cross3(u, ref, axis);
    double normAxis = sqrt(dot3(axis, axis));
    if (normAxis < tol) {
        if (fabs(dot3(u, ref) - 1.0) < tol) {
            q[0] = 1.0; q[1] = 0.0; q[2] = 0.0; q[3] = 0.0;
            return 0;
        }
        return -1;
    }
    axis[0] /= normAxis; axis[1] /= normAxis; axis[2] /= normAxis;
    double cosAngle = sqrt(0.5 * (1 + dot3(u, ref)));
    double sinAngle = sqrt(1 - cosAngle * cosAngle);
    q[0] = cosAngle;
    q[1] = sinAngle * axis[0];
    q[2] = sinAngle * axis[1];
    q[3] = sinAngle * axis[2];
    return 0;
}

/* CoordinateSystemTrafo(origin, orientation) (CoordinateSystemTrafo.cpp:18-23) */
void sco_trafo_make(sco_trafo* t, const double* origin, const double* quat) {
    for (int i = 0; i < 3; ++i) t->origin[i] = origin[i];
    for (int i = 0; i < 4; ++i) t->quat[i] = quat[i];
    quat_rotmat(t->quat, t->M);
}
/* CoordinateSystemTrafo::invert (CoordinateSystemTrafo.cpp:25-29) */
void sco_trafo_invert(sco_trafo* t) {
    double r[3];
    quat_rotate(t->quat, t->origin, r);
    t->origin[0] = -r[0]; t->origin[1] = -r[1]; t->origin[2] = -r[2];
    t->quat[1] = -t->quat[1]; t->quat[2] = -t->quat[2]; t->quat[3] = -t->quat[3];
    double M[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i * 3 + j] = t->M[j * 3 + i];
    memcpy(t->M, M, sizeof(M));
}
/* CoordinateSystemTrafo::operator*= (CoordinateSystemTrafo.cpp:38-43) */
void sco_trafo_compose(sco_trafo* t, const sco_trafo* right) {
    double rc[4] = {right->quat[0], -right->quat[1], -right->quat[2], -right->quat[3]};
    double r[3];
    quat_rotate(rc, t->origin, r);
    t->origin[0] = r[0] + right->origin[0];
    t->origin[1] = r[1] + right->origin[1];
    t->origin[2] = r[2] + right->origin[2];
    double q[4];
    quat_mul(t->quat, right->quat, q);
    memcpy(t->quat, q, sizeof(q));
    quat_normalize(t->quat);
    quat_rotmat(t->quat, t->M);
}
/* transformTo / rotateTo (CoordinateSystemTrafo.h:77-85) */
static inline void trafo_transform_to(const sco_trafo* t, const double* r, double* out) {
    double d[3] = {r[0] - t->origin[0], r[1] - t->origin[1], r[2] - t->origin[2]};
    matvec(t->M, d, out);
}
static inline void trafo_rotate_to(const sco_trafo* t, const double* r, double* out) {
    matvec(t->M, r, out);
}

/* exported for the pinning tests against the reference's own
   CoordinateSystemTrafo::transformTo / rotateTo and Quaternion::rotate */
void sco_trafo_transform_to(const sco_trafo* t, const double* r, double* out) { trafo_transform_to(t, r, out); }
void sco_trafo_rotate_to(const sco_trafo* t, const double* r, double* out) { trafo_rotate_to(t, r, out); }
void sco_quat_rotate(const double* q, const double* v, double* out) { quat_rotate(q, v, out); }

/* ------------------------------------------------------------------------ */
/* pusher: BorisPusher.h:56-124 and the unit switches PartBunchBase.hpp:468-513 */
/* ------------------------------------------------------------------------ */
static inline void push_one(double* R, const double* P, double dt) {
    const double s = SCO_C * dt;
    double r0 = R[0] / s, r1 = R[1] / s, r2 = R[2] / s;
    double g = sqrt(1.0 + dot3(P, P));
    r0 += 0.5 * P[0] / g;
    r1 += 0.5 * P[1] / g;
    r2 += 0.5 * P[2] / g;
    R[0] = r0 * s; R[1] = r1 * s; R[2] = r2 * s;
}

static inline void kick_one(double* P, const double* Ef, const double* Bf, double dt,
                            double mass, double charge) {
    const double ke = 0.5 * dt * charge * SCO_C / mass;
    P[0] += ke * Ef[0]; P[1] += ke * Ef[1]; P[2] += ke * Ef[2];
    const double gamma = sqrt(1.0 + dot3(P, P));
    const double kt = 0.5 * dt * charge * SCO_C * SCO_C / (gamma * mass);
    double t[3] = {kt * Bf[0], kt * Bf[1], kt * Bf[2]};
    double w[3], c[3];
    cross3(P, t, c);
    w[0] = P[0] + c[0]; w[1] = P[1] + c[1]; w[2] = P[2] + c[2];
    const double ks = 2.0 / (1.0 + dot3(t, t));
    double s[3] = {ks * t[0], ks * t[1], ks * t[2]};
    cross3(w, s, c);
    P[0] += c[0]; P[1] += c[1]; P[2] += c[2];
    P[0] += ke * Ef[0]; P[1] += ke * Ef[1]; P[2] += ke * Ef[2];
}

void sco_push(long long n, double* R, const double* P, double dt) {
    SCO_PAR
    for (long long i = 0; i < n; ++i) push_one(R + 3 * i, P + 3 * i, dt);
}

void sco_kick(long long n, double* P, const double* Ef, const double* Bf, double dt,
              double mass, double charge) {
    SCO_PAR
    for (long long i = 0; i < n; ++i) kick_one(P + 3 * i, Ef + 3 * i, Bf + 3 * i, dt, mass, charge);
}

/* ------------------------------------------------------------------------ */
/* bunch statistics: getLocalBounds (PartBunchBase.hpp:1201-1219),            */
/* calcMoments (:2185-2259), calcBeamParameters (:1529-1614)                 */
/* ------------------------------------------------------------------------ */
void sco_bounds(long long n, const double* R, double* rmin, double* rmax) {
    if (n == 0) {
        for (int d = 0; d < 3; ++d) rmin[d] = rmax[d] = 0.0;
        return;
    }
    if (g_threads > 1 && n > 1) {
        /* min / max are exact: the split does not change the result */
        double lo[3] = {R[0], R[1], R[2]}, hi[3] = {R[0], R[1], R[2]};
#pragma omp parallel num_threads(g_threads)
        {
            double tl[3] = {R[0], R[1], R[2]}, th[3] = {R[0], R[1], R[2]};
#pragma omp for schedule(static) nowait
            for (long long i = 1; i < n; ++i)
                for (int d = 0; d < 3; ++d) {
                    const double v = R[3 * i + d];
                    if (tl[d] > v) tl[d] = v;
                    else if (th[d] < v) th[d] = v;
                }
#pragma omp critical
            for (int d = 0; d < 3; ++d) {
                if (lo[d] > tl[d]) lo[d] = tl[d];
                if (hi[d] < th[d]) hi[d] = th[d];
            }
        }
        for (int d = 0; d < 3; ++d) { rmin[d] = lo[d]; rmax[d] = hi[d]; }
        return;
    }
    for (int d = 0; d < 3; ++d) rmin[d] = rmax[d] = R[d];
    for (long long i = 1; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
            if (rmin[d] > R[3 * i + d]) rmin[d] = R[3 * i + d];
            else if (rmax[d] < R[3 * i + d]) rmax[d] = R[3 * i + d];
        }
}

static void moments_range(long long k0, long long k1, const double* R, const double* P, double* m27);

/* 6 first moments + 21 second moments in OPAL's order (x,px,y,py,z,pz). */
static void moments_exact_range(long long k0, long long k1, const double* R, const double* P, sco_i128* acc) {
    for (int i = 0; i < 27; ++i) acc[i] = 0;
    double part[6];
    for (long long k = k0; k < k1; ++k) {
        part[1] = P[3 * k + 0]; part[3] = P[3 * k + 1]; part[5] = P[3 * k + 2];
        part[0] = R[3 * k + 0]; part[2] = R[3 * k + 1]; part[4] = R[3 * k + 2];
        int l = 6;
        for (int i = 0; i < 6; ++i) {
            acc[i] += ex_from(part[i]);
            for (int j = 0; j <= i; ++j) acc[l++] += ex_from(part[i] * part[j]);
        }
    }
}

void sco_moments(long long n, const double* R, const double* P, double* m27) {
    if (g_exact) {
        const int T = g_threads > 1 ? g_threads : 1;
        sco_i128* part = (sco_i128*)calloc((size_t)T * 27, sizeof(sco_i128));
#pragma omp parallel num_threads(T)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            moments_exact_range(n * t / T, n * (t + 1) / T, R, P, part + 27 * t);
        }
        for (int i = 0; i < 27; ++i) {
            sco_i128 a = 0;
            for (int t = 0; t < T; ++t) a += part[27 * t + i];
            m27[i] = ex_to_double(a);
        }
        free(part);
        return;
    }
    if (g_threads > 1) {
        const int T = g_threads;
        double* part = (double*)calloc((size_t)T * 27, sizeof(double));
#pragma omp parallel num_threads(T)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            const long long k0 = n * t / T, k1 = n * (t + 1) / T;
            moments_range(k0, k1, R, P, part + 27 * t);
        }
        for (int i = 0; i < 27; ++i) m27[i] = 0.0;
        for (int t = 0; t < T; ++t)
            for (int i = 0; i < 27; ++i) m27[i] += part[27 * t + i];
        free(part);
        return;
    }
    moments_range(0, n, R, P, m27);
}

static void moments_range(long long k0, long long k1, const double* R, const double* P, double* m27) {
    const long long n = k1;
    for (int i = 0; i < 27; ++i) m27[i] = 0.0;
    double part[6];
    for (long long k = k0; k < n; ++k) {
        part[1] = P[3 * k + 0]; part[3] = P[3 * k + 1]; part[5] = P[3 * k + 2];
        part[0] = R[3 * k + 0]; part[2] = R[3 * k + 1]; part[4] = R[3 * k + 2];
        int l = 6;
        for (int i = 0; i < 6; ++i) {
            m27[i] += part[i];
            for (int j = 0; j <= i; ++j) m27[l++] += part[i] * part[j];
        }
    }
}

double sco_sum_gamma(long long n, const double* P) {
    if (g_exact) {
        sco_i128 a = 0;
        for (long long i = 0; i < n; ++i) a += ex_from(sqrt(1.0 + dot3(P + 3 * i, P + 3 * i)));
        return ex_to_double(a);
    }
    double g = 0.0;
    for (long long i = 0; i < n; ++i) g += sqrt(1.0 + dot3(P + 3 * i, P + 3 * i));
    return g;
}

/* index of second moment (i,j), i>=j, in the m27 layout */
static int mom_idx(int i, int j) {
    if (i < j) { int t = i; i = j; j = t; }
    return 6 + i * (i + 1) / 2 + j;
}

/* calcBeamParameters from reduced sums: m27 (moments), sum of gamma, N. */
void sco_beam_parameters_from_sums(const double* m27, double gsum, double Nd, sco_beam_params* bp) {
    double N = Nd;
    double rsqsum[3], psqsum[3], rpsum[3], eps2[3];
    for (int i = 0; i < 3; ++i) {
        bp->rmean[i] = m27[2 * i] / N;
        bp->pmean[i] = m27[2 * i + 1] / N;
        rsqsum[i] = m27[mom_idx(2 * i, 2 * i)] - N * bp->rmean[i] * bp->rmean[i];
        psqsum[i] = m27[mom_idx(2 * i + 1, 2 * i + 1)] - N * bp->pmean[i] * bp->pmean[i];
        if (psqsum[i] < 0) psqsum[i] = 0;
        rpsum[i] = m27[mom_idx(2 * i, 2 * i + 1)] - N * bp->rmean[i] * bp->pmean[i];
    }
    for (int i = 0; i < 3; ++i) eps2[i] = (rsqsum[i] * psqsum[i] - rpsum[i] * rpsum[i]) / (N * N);
    for (int i = 0; i < 3; ++i) rpsum[i] /= N;
    for (int i = 0; i < 3; ++i) {
        bp->rrms[i] = sqrt(rsqsum[i] / N);
        bp->prms[i] = sqrt(psqsum[i] / N);
        bp->eps_norm[i] = sqrt(eps2[i] > 0.0 ? eps2[i] : 0.0);
        double tmp = bp->rrms[i] * bp->prms[i];
        double fac = (tmp == 0) ? 0.0 : 1.0 / tmp;
        bp->rprms[i] = rpsum[i] * fac;
    }
    double gamma = gsum / N;
    bp->gamma = gamma;
    double den = gamma * sqrt(1.0 - 1.0 / (gamma * gamma));
    for (int i = 0; i < 3; ++i) bp->eps[i] = bp->eps_norm[i] / den;
}

int sco_beam_parameters(long long n, const double* R, const double* P, sco_beam_params* bp) {
    memset(bp, 0, sizeof(*bp));
    sco_bounds(n, R, bp->rmin, bp->rmax);
    if (n == 0) return 0;
    double m27[27];
    sco_moments(n, R, P, m27);
    memcpy(bp->moments, m27, sizeof(m27));
    sco_beam_parameters_from_sums(m27, sco_sum_gamma(n, P), (double)n, bp);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* mesh (boundp): PartBunchBase.hpp:802-884                                   */
/* ------------------------------------------------------------------------ */
int sco_boundp(long long n, const double* R, const int* nr, double dh, sco_mesh* mesh) {
    double rmin[3], rmax[3];
    sco_bounds(n, R, rmin, rmax);
    for (int i = 0; i < 3; ++i) {
        double length = fabs(rmax[i] - rmin[i]);
        if (length < 1e-10) {
            rmax[i] += 1e-10;
            rmin[i] -= 1e-10;
        } else {
            rmax[i] += dh * length;
            rmin[i] -= dh * length;
        }
        mesh->hr[i] = (rmax[i] - rmin[i]) / (nr[i] - 1);
    }
    for (int i = 0; i < 3; ++i) {
        mesh->rmin[i] = rmin[i];
        mesh->rmax[i] = rmax[i];
        mesh->nr[i] = nr[i];
    }
    if (mesh->hr[0] * mesh->hr[1] * mesh->hr[2] <= 0) return SCO_ERR_MESH;
    mesh->origin[0] = rmin[0] - mesh->hr[0] / 2.0;
    mesh->origin[1] = rmin[1] - mesh->hr[1] / 2.0;
    mesh->origin[2] = rmin[2] - mesh->hr[2] / 2.0;
    return 0;
}

/* boundp of a DC beam (PartBunchBase.hpp:813-843 with dcBeam_m): x and y as
 * above, z not enlarged: rmax_z = rmin_z + periodLength, hr_z = periodLength
 * / (MT - 1). */
int sco_boundp_dc(long long n, const double* R, const int* nr, double dh, double period, sco_mesh* mesh) {
    double rmin[3], rmax[3];
    sco_bounds(n, R, rmin, rmax);
    for (int i = 0; i < 2; ++i) {
        double length = fabs(rmax[i] - rmin[i]);
        if (length < 1e-10) {
            rmax[i] += 1e-10;
            rmin[i] -= 1e-10;
        } else {
            rmax[i] += dh * length;
            rmin[i] -= dh * length;
        }
        mesh->hr[i] = (rmax[i] - rmin[i]) / (nr[i] - 1);
    }
    rmax[2] = rmin[2] + period;
    mesh->hr[2] = period / (nr[2] - 1);
    for (int i = 0; i < 3; ++i) {
        mesh->rmin[i] = rmin[i];
        mesh->rmax[i] = rmax[i];
        mesh->nr[i] = nr[i];
    }
    if (mesh->hr[0] * mesh->hr[1] * mesh->hr[2] <= 0) return SCO_ERR_MESH;
    mesh->origin[0] = rmin[0] - mesh->hr[0] / 2.0;
    mesh->origin[1] = rmin[1] - mesh->hr[1] / 2.0;
    mesh->origin[2] = rmin[2] - mesh->hr[2] / 2.0;
    return 0;
}

/* boundp's update() for a DC beam: the particle layout's domain follows the
 * mesh (RegionLayout::Repartition on the mesh's change notification,
 * RegionLayout.hpp:871-896; getMeshDomain :773-789: [origin, origin + h *
 * cells)), and ParticleSpatialLayout::update (ParticleSpatialLayout.hpp:
 * 296-297) applies ParticlePeriodicBCond (ParticleBConds.h:37-45) along z,
 * once per particle. */
void sco_wrap_z(long long n, double* R, const sco_mesh* m) {
    const double lo = m->origin[2];
    const double hi = m->origin[2] + m->hr[2] * (double)m->nr[2];
    SCO_PAR
    for (long long i = 0; i < n; ++i) {
        const double t = R[3 * i + 2];
        if (t < lo)
            R[3 * i + 2] = hi - (lo - t);
        else if (t >= hi)
            R[3 * i + 2] = lo + (t - hi);
    }
}

/* ------------------------------------------------------------------------ */
/* CIC (IntCIC.h:818-858 scatter, :935-975 gather)                           */
/* ------------------------------------------------------------------------ */
/* lower grid point and normalised offset; returns 0 when all 8 targets lie
 * inside the n^3 cell field, -1 otherwise (a guard-cell access).  With pz
 * (a DC beam) the z targets may also lie in the guard layer, planes -1 and
 * n: lower points -1 .. n-1 along z. */
static inline int cic_locate_bc(const sco_mesh* m, const double* x, int* lgp, double* dpos, int pz) {
    for (int d = 0; d < 3; ++d) {
        /* getVertexBelow (UniformCartesian.hpp:1025-1039) */
        int i = (int)((x[d] - m->origin[d]) / m->hr[d]);
        int ngp = (x[d] >= m->origin[d]) ? i : i - 1;
        /* getCellPosition (UniformCartesian.hpp:1084-1097) */
        double gpos = (ngp + 0.5) * m->hr[d] + m->origin[d];
        double delta = m->hr[d];
        if (gpos > x[d]) {
            lgp[d] = ngp - 1;
            gpos = gpos - delta;
        } else {
            lgp[d] = ngp;
        }
        dpos[d] = x[d] - gpos;
        dpos[d] /= delta;
        const int guard = (pz && d == 2) ? 1 : 0;
        if (lgp[d] < -guard || lgp[d] + 1 > m->nr[d] - 1 + guard) return -1;
    }
    return 0;
}
static inline int cic_locate(const sco_mesh* m, const double* x, int* lgp, double* dpos) {
    return cic_locate_bc(m, x, lgp, dpos, 0);
}

static int scatter_range(long long p0, long long p1, const double* R, double q, const sco_mesh* m, double* rho,
                         int pz);

static int scatter_bc(long long n, const double* R, double q, const sco_mesh* m, double* rho, int pz) {
    if (g_threads > 1) {
        const int T = g_threads;
        const long long M = (long long)m->nr[0] * m->nr[1] * m->nr[2];
        double* grids = (double*)calloc((size_t)T * M, sizeof(double));
        int bad = 0;
#pragma omp parallel num_threads(T) reduction(| : bad)
        {
#ifdef _OPENMP
            const int t = omp_get_thread_num();
#else
            const int t = 0;
#endif
            bad |= scatter_range(n * t / T, n * (t + 1) / T, R, q, m, grids + (size_t)t * M, pz) != 0;
        }
#pragma omp parallel for num_threads(T) schedule(static)
        for (long long c = 0; c < M; ++c)
            for (int t = 0; t < T; ++t) rho[c] += grids[(size_t)t * M + c];
        free(grids);
        return bad ? SCO_ERR_GUARD : 0;
    }
    return scatter_range(0, n, R, q, m, rho, pz);
}

int sco_scatter_cic(long long n, const double* R, double q, const sco_mesh* m, double* rho) {
    return scatter_bc(n, R, q, m, rho, 0);
}

/* The single-rank scatter of a DC beam: the charge IntCIC writes into the z
 * guard layer is not carried into the field (ParticleAttrib::scatter zeroes
 * the guard cells, ParticleAttrib.h:207-221, and accumGuardCells,
 * BareField.hpp:1013-1079, adds guard cells only into neighbouring local
 * fields, of which one vnode has none). */
int sco_scatter_cic_dc(long long n, const double* R, double q, const sco_mesh* m, double* rho) {
    return scatter_bc(n, R, q, m, rho, 1);
}

static int scatter_range(long long p0, long long p1, const double* R, double q, const sco_mesh* m, double* rho,
                         int pz) {
    const long long nx = m->nr[0], nxy = (long long)m->nr[0] * m->nr[1];
    const long long n = p1;
    int bad = 0;
    for (long long p = p0; p < n; ++p) {
        int l[3];
        double d[3];
        if (cic_locate_bc(m, R + 3 * p, l, d, pz)) { bad = 1; continue; }
        const long long b = l[0] + nx * l[1] + nxy * l[2];
        if (l[2] >= 0) { /* plane l: inside unless a DC beam's guard plane -1 */
            rho[b] += (1 - d[0]) * (1 - d[1]) * (1 - d[2]) * q;
            rho[b + 1] += d[0] * (1 - d[1]) * (1 - d[2]) * q;
            rho[b + nx] += (1 - d[0]) * d[1] * (1 - d[2]) * q;
            rho[b + nx + 1] += d[0] * d[1] * (1 - d[2]) * q;
        }
        if (l[2] + 1 < m->nr[2]) { /* plane l + 1: inside unless the guard plane n */
            rho[b + nxy] += (1 - d[0]) * (1 - d[1]) * d[2] * q;
            rho[b + nxy + 1] += d[0] * (1 - d[1]) * d[2] * q;
            rho[b + nxy + nx] += (1 - d[0]) * d[1] * d[2] * q;
            rho[b + nxy + nx + 1] += d[0] * d[1] * d[2] * q;
        }
    }
    return bad ? SCO_ERR_GUARD : 0;
}

/* E: 3 components per cell (interleaved).  Ef: 3 per particle.  With pz the
 * z guard planes hold the periodic images of the field (PeriodicFace, filled
 * before the gather, ParticleAttrib.h:297-299): plane n is plane 0 and plane
 * -1 is plane n-1. */
static int gather_bc(long long n, const double* R, const sco_mesh* m, const double* E, double* Ef, int pz) {
    const long long nx = m->nr[0], nxy = (long long)m->nr[0] * m->nr[1];
    const int n2 = m->nr[2];
    int bad = 0;
#pragma omp parallel for num_threads(g_threads) if(g_threads > 1) schedule(static) reduction(| : bad)
    for (long long p = 0; p < n; ++p) {
        int l[3];
        double d[3];
        if (cic_locate_bc(m, R + 3 * p, l, d, pz)) { bad = 1; Ef[3 * p] = Ef[3 * p + 1] = Ef[3 * p + 2] = 0.0; continue; }
        const int z0 = l[2] < 0 ? n2 - 1 : l[2];
        const int z1 = l[2] + 1 >= n2 ? 0 : l[2] + 1;
        const double* f = E + 3 * (l[0] + nx * l[1] + nxy * z0);
        const double w0 = (1 - d[0]) * (1 - d[1]) * (1 - d[2]);
        const double w1 = d[0] * (1 - d[1]) * (1 - d[2]);
        const double w2 = (1 - d[0]) * d[1] * (1 - d[2]);
        const double w3 = d[0] * d[1] * (1 - d[2]);
        const double w4 = (1 - d[0]) * (1 - d[1]) * d[2];
        const double w5 = d[0] * (1 - d[1]) * d[2];
        const double w6 = (1 - d[0]) * d[1] * d[2];
        const double w7 = d[0] * d[1] * d[2];
        const long long dz = 3 * nxy * (long long)(z1 - z0);
        const long long o1 = 3, o2 = 3 * nx, o3 = 3 * (nx + 1), o4 = dz, o5 = dz + 3,
                        o6 = dz + 3 * nx, o7 = dz + 3 * (nx + 1);
        for (int c = 0; c < 3; ++c) {
            Ef[3 * p + c] = w0 * f[c] + w1 * f[o1 + c] + w2 * f[o2 + c] + w3 * f[o3 + c] +
                            w4 * f[o4 + c] + w5 * f[o5 + c] + w6 * f[o6 + c] + w7 * f[o7 + c];
        }
    }
    return bad ? SCO_ERR_GUARD : 0;
}

int sco_gather_cic(long long n, const double* R, const sco_mesh* m, const double* E, double* Ef) {
    return gather_bc(n, R, m, E, Ef, 0);
}

int sco_gather_cic_dc(long long n, const double* R, const sco_mesh* m, const double* E, double* Ef) {
    return gather_bc(n, R, m, E, Ef, 1);
}

/* ------------------------------------------------------------------------ */
/* 1-D FFT engine with FFTPACK's interface (ippl/src/FFT/fftpack.h)           */
/* ------------------------------------------------------------------------ */
typedef void (*sco_init_fn)(size_t, double*);
typedef void (*sco_exec_fn)(size_t, double*, double*);
static sco_init_fn g_cffti, g_rffti;
static sco_exec_fn g_cfftf, g_cfftb, g_rfftf, g_rfftb;

/* project-written mixed-radix engine.  Work array layout (all doubles):
 *   [0] = n, [1..] = twiddles exp(-2 pi i k/n) for k < n (2n doubles),
 *   then 2n doubles of scratch.  Sizes agree with FFTPACK's (4n+15). */
static void own_cffti(size_t n, double* w) {
    w[0] = (double)n;
    for (size_t k = 0; k < n; ++k) {
        /* angle reduced to [0, pi/4]-friendly form by symmetry is not needed
         * at these lengths; libm cos/sin are within an ulp. */
        double a = -2.0 * SCO_PI * (double)k / (double)n;
        w[1 + 2 * k] = cos(a);
        w[2 + 2 * k] = sin(a);
    }
}

static void own_fft_rec(size_t n, const double* in, size_t is, double* out, int sign,
                        const double* tw, size_t ts, size_t N) {
    if (n == 1) {
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    size_t p;
    if (n % 4 == 0) p = 4;
    else if (n % 2 == 0) p = 2;
    else if (n % 3 == 0) p = 3;
    else if (n % 5 == 0) p = 5;
    else {
        p = n;
        for (size_t f = 7; f * f <= n; f += 2)
            if (n % f == 0) { p = f; break; }
    }
    size_t m = n / p;
    for (size_t q = 0; q < p; ++q) own_fft_rec(m, in + 2 * q * is, is * p, out + 2 * q * m, sign, tw, ts * p, N);
    double tre[64], tim[64], ore[64], oim[64];
    double* bre = tre; double* bim = tim; double* cre = ore; double* cim = oim;
    double* heap = NULL;
    if (p > 64) {
        heap = (double*)malloc(4 * p * sizeof(double));
        bre = heap; bim = heap + p; cre = heap + 2 * p; cim = heap + 3 * p;
    }
    for (size_t k = 0; k < m; ++k) {
        for (size_t q = 0; q < p; ++q) {
            size_t e = (q * k * ts) % N;
            double wr = tw[2 * e], wi = sign * tw[2 * e + 1];
            double yr = out[2 * (q * m + k)], yi = out[2 * (q * m + k) + 1];
            bre[q] = yr * wr - yi * wi;
            bim[q] = yr * wi + yi * wr;
        }
        for (size_t s = 0; s < p; ++s) {
            double sr = 0.0, si = 0.0;
            for (size_t q = 0; q < p; ++q) {
                size_t e = ((q * s) % p) * (N / p);
                double wr = tw[2 * e], wi = sign * tw[2 * e + 1];
                sr += bre[q] * wr - bim[q] * wi;
                si += bre[q] * wi + bim[q] * wr;
            }
            cre[s] = sr;
            cim[s] = si;
        }
        for (size_t s = 0; s < p; ++s) {
            out[2 * (k + s * m)] = cre[s];
            out[2 * (k + s * m) + 1] = cim[s];
        }
    }
    free(heap);
}

static void own_cfft(size_t n, double* c, double* w, int sign) {
    double* scratch = w + 1 + 2 * n;
    memcpy(scratch, c, 2 * n * sizeof(double));
    own_fft_rec(n, scratch, 1, c, sign, w + 1, 1, n);
}
static void own_cfftf(size_t n, double* c, double* w) { own_cfft(n, c, w, +1); }
static void own_cfftb(size_t n, double* c, double* w) { own_cfft(n, c, w, -1); }

/* real transforms through a complex transform of length n; output packed as
 * FFTPACK does: r0, (re1, im1), ..., and re_{n/2} last when n is even. */
static void own_rffti(size_t n, double* w) { own_cffti(n, w); }
static void own_rfftf(size_t n, double* r, double* w) {
    double* c = (double*)malloc(2 * n * sizeof(double));
    double* wk = (double*)malloc((1 + 4 * n) * sizeof(double));
    memcpy(wk, w, (1 + 2 * n) * sizeof(double));
    for (size_t i = 0; i < n; ++i) { c[2 * i] = r[i]; c[2 * i + 1] = 0.0; }
    own_cfft(n, c, wk, +1);
    r[0] = c[0];
    for (size_t k = 1; 2 * k < n; ++k) { r[2 * k - 1] = c[2 * k]; r[2 * k] = c[2 * k + 1]; }
    if (n % 2 == 0) r[n - 1] = c[n];
    free(c);
    free(wk);
}
static void own_rfftb(size_t n, double* r, double* w) {
    double* c = (double*)malloc(2 * n * sizeof(double));
    double* wk = (double*)malloc((1 + 4 * n) * sizeof(double));
    memcpy(wk, w, (1 + 2 * n) * sizeof(double));
    c[0] = r[0]; c[1] = 0.0;
    for (size_t k = 1; 2 * k < n; ++k) {
        c[2 * k] = r[2 * k - 1]; c[2 * k + 1] = r[2 * k];
        c[2 * (n - k)] = r[2 * k - 1]; c[2 * (n - k) + 1] = -r[2 * k];
    }
    if (n % 2 == 0) { c[n] = r[n - 1]; c[n + 1] = 0.0; }
    own_cfft(n, c, wk, -1);
    for (size_t i = 0; i < n; ++i) r[i] = c[2 * i];
    free(c);
    free(wk);
}

static int g_engine_is_own = 1;
static void engine_defaults(void) {
    if (!g_cffti) {
        g_cffti = own_cffti; g_cfftf = own_cfftf; g_cfftb = own_cfftb;
        g_rffti = own_rffti; g_rfftf = own_rfftf; g_rfftb = own_rfftb;
        g_engine_is_own = 1;
    }
}

void sco_set_fft_engine(void* cffti, void* cfftf, void* cfftb, void* rffti, void* rfftf, void* rfftb) {
    if (!cffti) {
        g_cffti = NULL;
        engine_defaults();
        return;
    }
    g_cffti = (sco_init_fn)cffti; g_cfftf = (sco_exec_fn)cfftf; g_cfftb = (sco_exec_fn)cfftb;
    g_rffti = (sco_init_fn)rffti; g_rfftf = (sco_exec_fn)rfftf; g_rfftb = (sco_exec_fn)rfftb;
    g_engine_is_own = 0;
}
int sco_fft_engine_is_own(void) { engine_defaults(); return g_engine_is_own; }

/* 1-D entry points with the engine's semantics (for tests) */
void sco_fft1d(int kind, long long n, double* data) {
    engine_defaults();
    double* w = (double*)calloc(4 * (size_t)n + 15 + 2 * (size_t)n + 8, sizeof(double));
    if (kind == 0) { g_cffti((size_t)n, w); g_cfftf((size_t)n, data, w); }
    else if (kind == 1) { g_cffti((size_t)n, w); g_cfftb((size_t)n, data, w); }
    else if (kind == 2) { g_rffti((size_t)n, w); g_rfftf((size_t)n, data, w); }
    else { g_rffti((size_t)n, w); g_rfftb((size_t)n, data, w); }
    free(w);
}

/* ------------------------------------------------------------------------ */
/* 3-D RC FFT on the doubled grid (FFT.hpp:1078-1340, :1483-1710).            */
/* Real field: L0*L1*L2, x fastest.  Spectrum: (L0/2+1)*L1*L2, kx fastest.    */
/* Forward: real-to-complex along x (FFTPACK forward + half-complex repack,   */
/* fftpack_FFT.h:218-240), then forward complex transforms along y and z.     */
/* Inverse: backward complex along z and y, then complex-to-real along x,     */
/* then multiply by normFact = 1/L0/L1/L2 (FFT.hpp:726-732, :1706).           */
/* ------------------------------------------------------------------------ */
typedef struct {
    double *wr, *w1, *w2, *strip;
} fft_ws;

static void fft_ws_init(fft_ws* w, long long L0, long long L1, long long L2) {
    w->wr = (double*)calloc(4 * L0 + 15 + 2 * L0 + 8, sizeof(double));
    w->w1 = (double*)calloc(4 * L1 + 15 + 2 * L1 + 8, sizeof(double));
    w->w2 = (double*)calloc(4 * L2 + 15 + 2 * L2 + 8, sizeof(double));
    long long Lmax = L0 > L1 ? L0 : L1;
    if (L2 > Lmax) Lmax = L2;
    w->strip = (double*)malloc((2 * Lmax + 4) * sizeof(double));
    g_rffti((size_t)L0, w->wr);
    g_cffti((size_t)L1, w->w1);
    g_cffti((size_t)L2, w->w2);
}

static void fft_ws_free(fft_ws* w) {
    free(w->wr); free(w->w1); free(w->w2); free(w->strip);
}

/* complex transforms of the columns along y (axis 1) or z (axis 2) */
static void fft_columns(double* spec, long long C0, long long L1, long long L2, int axis, int forward) {
    const long long outer = axis == 1 ? L2 : L1;
    const long long len = axis == 1 ? L1 : L2;
    const long long stride = axis == 1 ? C0 : C0 * L1;
#pragma omp parallel num_threads(g_threads) if(g_threads > 1)
    {
        fft_ws ws;
        fft_ws_init(&ws, 2, L1, L2);
        double* strip = ws.strip;
        double* w = axis == 1 ? ws.w1 : ws.w2;
#pragma omp for schedule(static)
        for (long long o = 0; o < outer; ++o) {
            const long long base = axis == 1 ? C0 * L1 * o : C0 * o;
            for (long long kx = 0; kx < C0; ++kx) {
                double* c = spec + 2 * (base + kx);
                for (long long e = 0; e < len; ++e) {
                    strip[2 * e] = c[2 * stride * e];
                    strip[2 * e + 1] = c[2 * stride * e + 1];
                }
                if (forward) g_cfftf((size_t)len, strip, w);
                else g_cfftb((size_t)len, strip, w);
                for (long long e = 0; e < len; ++e) {
                    c[2 * stride * e] = strip[2 * e];
                    c[2 * stride * e + 1] = strip[2 * e + 1];
                }
            }
        }
        fft_ws_free(&ws);
    }
}

void sco_fft3d_r2c(const int* L, const double* in, double* out) {
    engine_defaults();
    const long long L0 = L[0], L1 = L[1], L2 = L[2], C0 = L0 / 2 + 1;
#pragma omp parallel num_threads(g_threads) if(g_threads > 1)
    {
        fft_ws ws;
        fft_ws_init(&ws, L0, 2, 2);
        double* strip = ws.strip;
#pragma omp for schedule(static)
        for (long long r = 0; r < L1 * L2; ++r) {
            memcpy(strip, in + L0 * r, L0 * sizeof(double));
            g_rfftf((size_t)L0, strip, ws.wr);
            double* o = out + 2 * C0 * r;
            o[0] = strip[0]; o[1] = 0.0;
            for (long long m = 1; 2 * m < L0; ++m) { o[2 * m] = strip[2 * m - 1]; o[2 * m + 1] = strip[2 * m]; }
            if (L0 % 2 == 0) { o[2 * (C0 - 1)] = strip[L0 - 1]; o[2 * (C0 - 1) + 1] = 0.0; }
        }
        fft_ws_free(&ws);
    }
    fft_columns(out, C0, L1, L2, 1, 1);
    fft_columns(out, C0, L1, L2, 2, 1);
}

/* inverse; `spec` is overwritten. `out` receives the normalised real field. */
void sco_fft3d_c2r(const int* L, double* spec, double* out) {
    engine_defaults();
    const long long L0 = L[0], L1 = L[1], L2 = L[2], C0 = L0 / 2 + 1;
    fft_columns(spec, C0, L1, L2, 2, 0);
    fft_columns(spec, C0, L1, L2, 1, 0);
    double normFact = 1.0;
    normFact /= L0;
    normFact /= L1;
    normFact /= L2;
#pragma omp parallel num_threads(g_threads) if(g_threads > 1)
    {
        fft_ws ws;
        fft_ws_init(&ws, L0, 2, 2);
        double* strip = ws.strip;
#pragma omp for schedule(static)
        for (long long r = 0; r < L1 * L2; ++r) {
            const double* c = spec + 2 * C0 * r;
            /* netlib repack (fftpack_FFT.h:229-233) */
            strip[0] = c[0];
            for (long long m = 1; 2 * m < L0; ++m) { strip[2 * m - 1] = c[2 * m]; strip[2 * m] = c[2 * m + 1]; }
            if (L0 % 2 == 0) strip[L0 - 1] = c[2 * (C0 - 1)];
            g_rfftb((size_t)L0, strip, ws.wr);
            double* o = out + L0 * r;
            for (long long i = 0; i < L0; ++i) o[i] = strip[i] * normFact;
        }
        fft_ws_free(&ws);
    }
}

/* ------------------------------------------------------------------------ */
/* integrated Green's function (FFTPoissonSolver.cpp:459-522) and mirror     */
/* (:641-664).  Output: doubled real grid G2, (2nx)(2ny)(2nz), x fastest.     */
/* The plane at index n of each axis is read from outside tmpgreen's domain   */
/* in the reference and never reaches the physical n^3 block of phi; here it  */
/* holds the value of the same closed form.                                   */
/* ------------------------------------------------------------------------ */
/* Elementary functions of the antiderivative.  By default the host libm,
 * as the reference calls std::atan / std::log.  In exact mode they are
 * evaluated in quad precision (libquadmath) and rounded once, i.e. correctly
 * rounded: the field then no longer depends on which libm rounds which
 * argument (the eight-corner difference turns a one-ulp change of one value
 * into ~1e-11 of the field). */
static double igf_atan(double v) { return g_exact ? (double)atanq((__float128)v) : atan(v); }
static double igf_log(double v) { return g_exact ? (double)logq((__float128)v) : log(v); }

static double igf_antiderivative(double x, double y, double z, double cellVolume) {
    double r = sqrt(x * x + y * y + z * z);
    double tmpgrn = -z * z * igf_atan(x * y / (z * r)) / 2;
    tmpgrn += -y * y * igf_atan(x * z / (y * r)) / 2;
    tmpgrn += -x * x * igf_atan(y * z / (x * r)) / 2;
    tmpgrn += y * z * igf_log(x + r);
    tmpgrn += x * z * igf_log(y + r);
    tmpgrn += x * y * igf_log(z + r);
    return tmpgrn / cellVolume;
}

void sco_igf(const int* nr, const double* hr, double* G2) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const long long t0 = n0 + 2, t1 = n1 + 2, t2 = n2 + 2;
    const long long L0 = 2 * n0, L1 = 2 * n1, L2 = 2 * n2;
    double cellVolume = hr[0] * hr[1] * hr[2];
    double* tmp = (double*)malloc(t0 * t1 * t2 * sizeof(double));
    SCO_PAR
    for (long long k = 0; k < t2; ++k)
        for (long long j = 0; j < t1; ++j)
            for (long long i = 0; i < t0; ++i) {
                double vx = i * hr[0] - hr[0] / 2;
                double vy = j * hr[1] - hr[1] / 2;
                double vz = k * hr[2] - hr[2] / 2;
                tmp[i + t0 * (j + t1 * k)] = igf_antiderivative(vx, vy, vz, cellVolume);
            }
#define TG(a, b, c) tmp[(a) + t0 * ((b) + t1 * (c))]
    memset(G2, 0, L0 * L1 * L2 * sizeof(double));
    SCO_PAR
    for (long long k = 0; k <= n2; ++k)
        for (long long j = 0; j <= n1; ++j)
            for (long long i = 0; i <= n0; ++i) {
                double g = TG(i + 1, j + 1, k + 1);
                g += TG(i + 1, j, k);
                g += TG(i, j + 1, k);
                g += TG(i, j, k + 1);
                g -= TG(i + 1, j + 1, k);
                g -= TG(i + 1, j, k + 1);
                g -= TG(i, j + 1, k + 1);
                g -= TG(i, j, k);
                if (i < L0 && j < L1 && k < L2) G2[i + L0 * (j + L1 * k)] = g;
            }
#undef TG
    free(tmp);
    /* mirrorRhoField: G[0,0,0] <- G[0,0,1]; then mirror x, y, z in turn */
    G2[0] = G2[L0 * L1 * 1];
    for (long long k = 0; k <= n2 && k < L2; ++k)
        for (long long j = 0; j <= n1 && j < L1; ++j)
            for (long long i = n0 + 1; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[(L0 - i) + L0 * (j + L1 * k)];
    for (long long k = 0; k <= n2 && k < L2; ++k)
        for (long long j = n1 + 1; j < L1; ++j)
            for (long long i = 0; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[i + L0 * ((L1 - j) + L1 * k)];
    for (long long k = n2 + 1; k < L2; ++k)
        for (long long j = 0; j < L1; ++j)
            for (long long i = 0; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[i + L0 * (j + L1 * (L2 - k))];
}

/* ------------------------------------------------------------------------ */
/* FFTPoissonSolver::computePotential(rho, hr)  (FFTPoissonSolver.cpp:337-382) */
/* rho: n^3, x fastest; overwritten by the convolution (without the later    */
/* cell-volume and coupling factors, which computeSelfFields applies).       */
/* ------------------------------------------------------------------------ */
int sco_compute_potential(const int* nr, double* rho, const double* hr) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const int L[3] = {2 * nr[0], 2 * nr[1], 2 * nr[2]};
    const long long L0 = L[0], L1 = L[1], L2 = L[2], C0 = L0 / 2 + 1;
    const long long D = L0 * L1 * L2, S = C0 * L1 * L2;
    double* rho2 = (double*)calloc(D, sizeof(double));
    double* rhot = (double*)malloc(2 * S * sizeof(double));
    double* grnt = (double*)malloc(2 * S * sizeof(double));
    double* G2 = (double*)malloc(D * sizeof(double));
    if (!rho2 || !rhot || !grnt || !G2) { free(rho2); free(rhot); free(grnt); free(G2); return SCO_ERR_OOM; }
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            memcpy(rho2 + L0 * (j + L1 * k), rho + n0 * (j + n1 * k), n0 * sizeof(double));
    sco_fft3d_r2c(L, rho2, rhot);
    sco_igf(nr, hr, G2);
    sco_fft3d_r2c(L, G2, grnt);
    for (long long s = 0; s < S; ++s) {
        double ar = rhot[2 * s], ai = rhot[2 * s + 1], br = grnt[2 * s], bi = grnt[2 * s + 1];
        rhot[2 * s] = ar * br - ai * bi;
        rhot[2 * s + 1] = ar * bi + ai * br;
    }
    sco_fft3d_c2r(L, rhot, rho2);
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            memcpy(rho + n0 * (j + n1 * k), rho2 + L0 * (j + L1 * k), n0 * sizeof(double));
    free(rho2); free(rhot); free(grnt); free(G2);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* -Grad (UniformCartesian.hpp:2129-2203) with PartBunch.cpp:573-575 scaling */
/* phi: n^3; E: 3*n^3 interleaved.  h: unscaled mesh spacing.                */
/* ------------------------------------------------------------------------ */
void sco_neg_grad_scaled(const int* nr, const double* phi, const double* h, double gammaz, double* E) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const double id[3] = {0.5 / h[0], 0.5 / h[1], 0.5 / h[2]};
    const long long st[3] = {1, n0, n0 * n1};
    const long long nn[3] = {n0, n1, n2};
    const double sc[3] = {gammaz / 1.0, gammaz / 1.0, 1.0 / (1.0 * gammaz)};
    SCO_PAR
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            for (long long i = 0; i < n0; ++i) {
                const long long c = i + n0 * (j + n1 * k);
                const long long idx[3] = {i, j, k};
                for (int d = 0; d < 3; ++d) {
                    double g;
                    const double* f = phi + c;
                    const long long s = st[d];
                    if (idx[d] == 0) {
                        g = id[d] * (-1.0 * f[2 * s] + 4.0 * f[s] - 3.0 * f[0]);
                    } else if (idx[d] == nn[d] - 1) {
                        g = id[d] * (1.0 * f[-2 * s] - 4.0 * f[-s] + 3.0 * f[0]);
                    } else {
                        g = id[d] * (f[s] - f[-s]);
                    }
                    E[3 * c + d] = (-g) * sc[d];
                }
            }
}

/* ------------------------------------------------------------------------ */
/* PartBunch::computeSelfFields()  (PartBunch.cpp:482-647) on a bunch that is */
/* already in the beam frame, preceded by boundp (PartBunchBase.hpp:802-884). */
/* ------------------------------------------------------------------------ */
int sco_compute_self_fields(const sco_params* prm, double* Q, long long n, double* R,
                            const double* P, double* Ef, double* Bf, sco_debug* dbg) {
    sco_mesh mesh;
    const int dc = prm->period > 0.0;
    int rc = dc ? sco_boundp_dc(n, R, prm->nr, prm->dh, prm->period, &mesh) : sco_boundp(n, R, prm->nr, prm->dh, &mesh);
    if (rc) return rc;
    if (dc) sco_wrap_z(n, R, &mesh);
    const long long n0 = prm->nr[0], n1 = prm->nr[1], n2 = prm->nr[2];
    const long long M = n0 * n1 * n2;
    double* rho = (double*)calloc(M, sizeof(double));
    double* E = (double*)malloc(3 * M * sizeof(double));
    if (!rho || !E) { free(rho); free(E); return SCO_ERR_OOM; }
    const double dt = prm->dT;
    /* Q *= dt; Q.scatter(rho, R, CIC); Q /= dt; rho /= dT   (:493-496) */
    double qdt = *Q * dt;
    rc = dc ? sco_scatter_cic_dc(n, R, qdt, &mesh, rho) : sco_scatter_cic(n, R, qdt, &mesh, rho);
    *Q = qdt / dt;
    if (rc) { free(rho); free(E); return rc; }
    SCO_PAR
    for (long long c = 0; c < M; ++c) rho[c] /= prm->dT;
    /* gamma_z from the mean longitudinal momentum (:499-502) */
    double psum2 = 0.0;
    if (g_threads > 1 || g_exact) {
        double m27[27];
        sco_moments(n, R, P, m27); /* thread-ordered partial sums; pz sum is m27[5] */
        psum2 = m27[5];
    } else {
        for (long long i = 0; i < n; ++i) psum2 += P[3 * i + 2];
    }
    double gammaz = psum2 / (double)n;
    gammaz *= gammaz;
    gammaz = sqrt(gammaz + 1.0);
    double hr_scaled[3] = {mesh.hr[0] * 1.0, mesh.hr[1] * 1.0, mesh.hr[2] * 1.0};
    hr_scaled[2] *= gammaz;
    double tmp2 = 1 / hr_scaled[0] * 1 / hr_scaled[1] * 1 / hr_scaled[2];
    SCO_PAR
    for (long long c = 0; c < M; ++c) rho[c] *= tmp2;
    if (dbg && dbg->rho) memcpy(dbg->rho, rho, M * sizeof(double));
    rc = dc ? sco_compute_potential_periodic_z(prm->nr, rho, hr_scaled) : sco_compute_potential(prm->nr, rho, hr_scaled);
    if (rc) { free(rho); free(E); return rc; }
    const double hvol = hr_scaled[0] * hr_scaled[1] * hr_scaled[2];
    SCO_PAR
    for (long long c = 0; c < M; ++c) rho[c] *= hvol;
    SCO_PAR
    for (long long c = 0; c < M; ++c) rho[c] *= prm->coupling;
    if (dbg && dbg->phi) memcpy(dbg->phi, rho, M * sizeof(double));
    sco_neg_grad_scaled(prm->nr, rho, mesh.hr, gammaz, E);
    if (dbg && dbg->E) memcpy(dbg->E, E, 3 * M * sizeof(double));
    rc = dc ? sco_gather_cic_dc(n, R, &mesh, E, Ef) : sco_gather_cic(n, R, &mesh, E, Ef);
    const double betaC = sqrt(gammaz * gammaz - 1.0) / gammaz / SCO_C;
    SCO_PAR
    for (long long i = 0; i < n; ++i) {
        Bf[3 * i + 0] = 0.0 - betaC * Ef[3 * i + 1];
        Bf[3 * i + 1] = 0.0 + betaC * Ef[3 * i + 0];
        Bf[3 * i + 2] = 0.0;
    }
    if (dbg) {
        dbg->mesh = mesh;
        dbg->gammaz = gammaz;
        dbg->hr_scaled[0] = hr_scaled[0];
        dbg->hr_scaled[1] = hr_scaled[1];
        dbg->hr_scaled[2] = hr_scaled[2];
    }
    free(rho);
    free(E);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* periodic z (FFTPoissonSolver with bcz = "PERIODIC", FFTPoissonSolver.cpp:  */
/* 60, :130-155, :189-190, :661-662): the grid is doubled in x and y only;     */
/* G is the integrated Green's function at offsets k in [0, nz) along z,      */
/* mirrored in x and y but not in z, with G[0,0,0] <- G[0,0,1]; the          */
/* convolution is cyclic along z.  G2: (2nx)(2ny)(nz), x fastest.            */
/* ------------------------------------------------------------------------ */
void sco_igf_periodic_z(const int* nr, const double* hr, double* G2) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const long long t0 = n0 + 2, t1 = n1 + 2, t2 = n2 + 2;
    const long long L0 = 2 * n0, L1 = 2 * n1, L2 = n2;
    double cellVolume = hr[0] * hr[1] * hr[2];
    double* tmp = (double*)malloc(t0 * t1 * t2 * sizeof(double));
    SCO_PAR
    for (long long k = 0; k < t2; ++k)
        for (long long j = 0; j < t1; ++j)
            for (long long i = 0; i < t0; ++i) {
                double vx = i * hr[0] - hr[0] / 2;
                double vy = j * hr[1] - hr[1] / 2;
                double vz = k * hr[2] - hr[2] / 2;
                tmp[i + t0 * (j + t1 * k)] = igf_antiderivative(vx, vy, vz, cellVolume);
            }
#define TG(a, b, c) tmp[(a) + t0 * ((b) + t1 * (c))]
    memset(G2, 0, L0 * L1 * L2 * sizeof(double));
    SCO_PAR
    for (long long k = 0; k < L2; ++k)
        for (long long j = 0; j <= n1; ++j)
            for (long long i = 0; i <= n0; ++i) {
                double g = TG(i + 1, j + 1, k + 1);
                g += TG(i + 1, j, k);
                g += TG(i, j + 1, k);
                g += TG(i, j, k + 1);
                g -= TG(i + 1, j + 1, k);
                g -= TG(i + 1, j, k + 1);
                g -= TG(i, j + 1, k + 1);
                g -= TG(i, j, k);
                if (i < L0 && j < L1) G2[i + L0 * (j + L1 * k)] = g;
            }
#undef TG
    free(tmp);
    if (L2 > 1) G2[0] = G2[L0 * L1 * 1];
    for (long long k = 0; k < L2; ++k)
        for (long long j = 0; j <= n1 && j < L1; ++j)
            for (long long i = n0 + 1; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[(L0 - i) + L0 * (j + L1 * k)];
    for (long long k = 0; k < L2; ++k)
        for (long long j = n1 + 1; j < L1; ++j)
            for (long long i = 0; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[i + L0 * ((L1 - j) + L1 * k)];
}

int sco_compute_potential_periodic_z(const int* nr, double* rho, const double* hr) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const int L[3] = {2 * nr[0], 2 * nr[1], nr[2]};
    const long long L0 = L[0], L1 = L[1], L2 = L[2], C0 = L0 / 2 + 1;
    const long long D = L0 * L1 * L2, S = C0 * L1 * L2;
    double* rho2 = (double*)calloc(D, sizeof(double));
    double* rhot = (double*)malloc(2 * S * sizeof(double));
    double* grnt = (double*)malloc(2 * S * sizeof(double));
    double* G2 = (double*)malloc(D * sizeof(double));
    if (!rho2 || !rhot || !grnt || !G2) { free(rho2); free(rhot); free(grnt); free(G2); return SCO_ERR_OOM; }
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            memcpy(rho2 + L0 * (j + L1 * k), rho + n0 * (j + n1 * k), n0 * sizeof(double));
    sco_fft3d_r2c(L, rho2, rhot);
    sco_igf_periodic_z(nr, hr, G2);
    sco_fft3d_r2c(L, G2, grnt);
    for (long long s = 0; s < S; ++s) {
        double ar = rhot[2 * s], ai = rhot[2 * s + 1], br = grnt[2 * s], bi = grnt[2 * s + 1];
        rhot[2 * s] = ar * br - ai * bi;
        rhot[2 * s + 1] = ar * bi + ai * br;
    }
    sco_fft3d_c2r(L, rhot, rho2);
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            memcpy(rho + n0 * (j + n1 * k), rho2 + L0 * (j + L1 * k), n0 * sizeof(double));
    free(rho2); free(rhot); free(grnt); free(G2);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* shifted integrated Green's function for the image charge                  */
/* (FFTPoissonSolver::shiftedIntGreensFunction, FFTPoissonSolver.cpp:546-639, */
/* and mirrorRhoField(ggrn2), :667-693).  Output: doubled real grid G2,        */
/* (2nx)(2ny)(2nz), x fastest.  Along z the grid is not mirrored: indices     */
/* k <= nz hold the offsets k (antiderivative planes at k hz - hz/2 + zshift), */
/* indices nz < k < 2nz the offsets k - 2nz (planes shifted by -nz hz).  No   */
/* G[0,0,0] overwrite.  The planes at index n of x and y are, as in sco_igf,  */
/* the closed form (the reference reads them outside tmpgreen's domain; they  */
/* never reach the physical block of phi).                                    */
/* ------------------------------------------------------------------------ */
void sco_igf_shifted(const int* nr, const double* hr, double zshift, double* G2) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const long long t0 = n0 + 2, t1 = n1 + 2, t2 = n2 + 2;
    const long long L0 = 2 * n0, L1 = 2 * n1, L2 = 2 * n2;
    double cellVolume = hr[0] * hr[1] * hr[2];
    double* ta = (double*)malloc(t0 * t1 * t2 * sizeof(double));
    double* tb = (double*)malloc(t0 * t1 * t2 * sizeof(double));
    SCO_PAR
    for (long long k = 0; k < t2; ++k)
        for (long long j = 0; j < t1; ++j)
            for (long long i = 0; i < t0; ++i) {
                double vx = i * hr[0] - hr[0] / 2;
                double vy = j * hr[1] - hr[1] / 2;
                double vz = k * hr[2] - hr[2] / 2 + zshift;
                ta[i + t0 * (j + t1 * k)] = igf_antiderivative(vx, vy, vz, cellVolume);
                vz = k * hr[2] - hr[2] / 2 + zshift - n2 * hr[2];
                tb[i + t0 * (j + t1 * k)] = igf_antiderivative(vx, vy, vz, cellVolume);
            }
#define CORNERS(T, a, b, c)                                                                     \
    (((((((T[(a + 1) + t0 * ((b + 1) + t1 * (c + 1))] + T[(a + 1) + t0 * ((b) + t1 * (c))]) + \
          T[(a) + t0 * ((b + 1) + t1 * (c))]) +                                                 \
         T[(a) + t0 * ((b) + t1 * (c + 1))]) -                                                  \
        T[(a + 1) + t0 * ((b + 1) + t1 * (c))]) -                                               \
       T[(a + 1) + t0 * ((b) + t1 * (c + 1))]) -                                                \
      T[(a) + t0 * ((b + 1) + t1 * (c + 1))]) -                                                 \
     T[(a) + t0 * ((b) + t1 * (c))])
    memset(G2, 0, L0 * L1 * L2 * sizeof(double));
    SCO_PAR
    for (long long k = 0; k < L2; ++k)
        for (long long j = 0; j <= n1; ++j)
            for (long long i = 0; i <= n0; ++i) {
                if (i >= L0 || j >= L1) continue;
                /* rho2[I][J][K] from tmpgreen (k <= nz), rho2[I][J][KE] = ggrn2[I][J][KE - nz] */
                const double g = k <= n2 ? CORNERS(ta, i, j, k) : CORNERS(tb, i, j, k - n2);
                G2[i + L0 * (j + L1 * k)] = g;
            }
#undef CORNERS
    free(ta);
    free(tb);
    /* rho2[IE][J][aK] = rho2[2nx - IE][J][aK]; rho2[aI][JE][aK] = rho2[aI][2ny - JE][aK] */
    for (long long k = 0; k < L2; ++k)
        for (long long j = 0; j <= n1 && j < L1; ++j)
            for (long long i = n0 + 1; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[(L0 - i) + L0 * (j + L1 * k)];
    for (long long k = 0; k < L2; ++k)
        for (long long j = n1 + 1; j < L1; ++j)
            for (long long i = 0; i < L0; ++i)
                G2[i + L0 * (j + L1 * k)] = G2[i + L0 * ((L1 - j) + L1 * k)];
}

/* ------------------------------------------------------------------------ */
/* FFTPoissonSolver::computePotential(rho, hr, zshift)  (FFTPoissonSolver.cpp: */
/* 287-327): the potential of the image charge.  imgrho2tr = -rho2tr * grntr; */
/* the inverse transform is read back with z flipped,                         */
/* rho[i][j][k] = rho2[i][j][nz - k - 1].                                     */
/* ------------------------------------------------------------------------ */
int sco_compute_potential_shifted(const int* nr, double* rho, const double* hr, double zshift) {
    const long long n0 = nr[0], n1 = nr[1], n2 = nr[2];
    const int L[3] = {2 * nr[0], 2 * nr[1], 2 * nr[2]};
    const long long L0 = L[0], L1 = L[1], L2 = L[2], C0 = L0 / 2 + 1;
    const long long D = L0 * L1 * L2, S = C0 * L1 * L2;
    double* rho2 = (double*)calloc(D, sizeof(double));
    double* rhot = (double*)malloc(2 * S * sizeof(double));
    double* grnt = (double*)malloc(2 * S * sizeof(double));
    double* G2 = (double*)malloc(D * sizeof(double));
    if (!rho2 || !rhot || !grnt || !G2) { free(rho2); free(rhot); free(grnt); free(G2); return SCO_ERR_OOM; }
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            memcpy(rho2 + L0 * (j + L1 * k), rho + n0 * (j + n1 * k), n0 * sizeof(double));
    sco_fft3d_r2c(L, rho2, rhot);
    sco_igf_shifted(nr, hr, zshift, G2);
    sco_fft3d_r2c(L, G2, grnt);
    for (long long s = 0; s < S; ++s) {
        double ar = rhot[2 * s], ai = rhot[2 * s + 1], br = grnt[2 * s], bi = grnt[2 * s + 1];
        rhot[2 * s] = -(ar * br - ai * bi);
        rhot[2 * s + 1] = -(ar * bi + ai * br);
    }
    sco_fft3d_c2r(L, rhot, rho2);
    for (long long k = 0; k < n2; ++k)
        for (long long j = 0; j < n1; ++j)
            memcpy(rho + n0 * (j + n1 * k), rho2 + L0 * (j + L1 * (n2 - k - 1)), n0 * sizeof(double));
    free(rho2); free(rhot); free(grnt); free(G2);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* energy bins: calcGammas (PartBunchBase.hpp:639-683): the mean of           */
/* sqrt(1 + P.P) over the particles of each bin, 1 for an empty bin.          */
/* ------------------------------------------------------------------------ */
int sco_bin_gammas(long long n, const double* P, const int* bin, int nbins, double* gamma, long long* count) {
    if (nbins <= 0) return SCO_ERR_ARG;
    for (long long i = 0; i < n; ++i)
        if (bin[i] < 0 || bin[i] >= nbins) return SCO_ERR_ARG;
    for (int b = 0; b < nbins; ++b) count[b] = 0;
    if (g_exact) {
        sco_i128* a = (sco_i128*)calloc(nbins, sizeof(sco_i128));
        if (!a) return SCO_ERR_OOM;
        for (long long i = 0; i < n; ++i) {
            a[bin[i]] += ex_from(sqrt(1.0 + dot3(P + 3 * i, P + 3 * i)));
            count[bin[i]] += 1;
        }
        for (int b = 0; b < nbins; ++b) gamma[b] = ex_to_double(a[b]);
        free(a);
    } else {
        for (int b = 0; b < nbins; ++b) gamma[b] = 0.0;
        for (long long i = 0; i < n; ++i) {
            gamma[bin[i]] += sqrt(1.0 + dot3(P + 3 * i, P + 3 * i));
            count[bin[i]] += 1;
        }
    }
    for (int b = 0; b < nbins; ++b) {
        if (count[b] != 0)
            gamma[b] /= (double)count[b];
        else
            gamma[b] = 1.0;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* The energy-bin loop of computeSpaceChargeFields (ParallelTTracker.cpp:567- */
/* 578) with PartBunch::computeSelfFields(int bin) (PartBunch.cpp:138-430) on */
/* a bunch already in the beam frame, preceded by boundp.  The charge of bin  */
/* b's particles is qi (setBinCharge, PartBunchBase.hpp:722-725), all other   */
/* particles carry none; Q is restored after every bin, so qi is unchanged.   */
/* Ef, Bf are accumulated from zero: per bin the field of the bin's charge    */
/* and of its image (a mirror charge behind the cathode plane, moving the     */
/* other way, hence the opposite sign of its magnetic field).  bin_gamma      */
/* (optional, nbins doubles) receives calcGammas' result.                     */
/* ------------------------------------------------------------------------ */
int sco_compute_self_fields_binned(const sco_params* prm, double qi, long long n, const double* R,
                                   const double* P, const int* bin, int nbins, int last_emitted,
                                   double* Ef, double* Bf, double* bin_gamma, sco_debug* dbg) {
    sco_mesh mesh;
    if (prm->period > 0.0) return SCO_ERR_ARG; /* energy bins with a DC beam: not a reference configuration */
    int rc = sco_boundp(n, R, prm->nr, prm->dh, &mesh);
    if (rc) return rc;
    const long long n0 = prm->nr[0], n1 = prm->nr[1], n2 = prm->nr[2];
    const long long M = n0 * n1 * n2;
    double* gam = (double*)malloc((nbins > 0 ? nbins : 1) * sizeof(double));
    long long* cnt = (long long*)malloc((nbins > 0 ? nbins : 1) * sizeof(long long));
    double* rho = (double*)malloc(M * sizeof(double));
    double* img = (double*)malloc(M * sizeof(double));
    double* E = (double*)malloc(3 * M * sizeof(double));
    double* Et = (double*)malloc(3 * n * sizeof(double));
    double* Rb = (double*)malloc(3 * n * sizeof(double));
    if (!gam || !cnt || !rho || !img || !E || !Et || !Rb) {
        rc = SCO_ERR_OOM;
        goto done;
    }
    /* calcGammas (:568) */
    rc = sco_bin_gammas(n, P, bin, nbins, gam, cnt);
    if (rc) goto done;
    if (bin_gamma) memcpy(bin_gamma, gam, nbins * sizeof(double));
    memset(Ef, 0, 3 * n * sizeof(double));
    memset(Bf, 0, 3 * n * sizeof(double));
    for (int b = 0; b < last_emitted && b < nbins; ++b) {
        /* setBinCharge(b); Q *= dt; scatter; Q /= dt; rho /= dT  (:153-170) */
        long long nb = 0;
        for (long long i = 0; i < n; ++i)
            if (bin[i] == b) {
                memcpy(Rb + 3 * nb, R + 3 * i, 3 * sizeof(double));
                ++nb;
            }
        memset(rho, 0, M * sizeof(double));
        const double qdt = qi * prm->dT;
        rc = sco_scatter_cic(nb, Rb, qdt, &mesh, rho);
        if (rc) goto done;
        for (long long c = 0; c < M; ++c) rho[c] /= prm->dT;
        /* (:173-185) */
        const double scaleFactor = 1;
        const double gammaz = gam[b];
        const double tmp2 = 1 / mesh.hr[0] * 1 / mesh.hr[1] * 1 / mesh.hr[2] /
                            (scaleFactor * scaleFactor * scaleFactor) / gammaz;
        for (long long c = 0; c < M; ++c) rho[c] *= tmp2;
        double hr_scaled[3] = {mesh.hr[0] * scaleFactor, mesh.hr[1] * scaleFactor, mesh.hr[2] * scaleFactor};
        hr_scaled[2] *= gammaz;
        memcpy(img, rho, M * sizeof(double));
        /* the bin's own field (:190-244) */
        rc = sco_compute_potential(prm->nr, rho, hr_scaled);
        if (rc) goto done;
        const double hvol = hr_scaled[0] * hr_scaled[1] * hr_scaled[2];
        for (long long c = 0; c < M; ++c) rho[c] *= hvol;
        for (long long c = 0; c < M; ++c) rho[c] *= prm->coupling;
        sco_neg_grad_scaled(prm->nr, rho, mesh.hr, gammaz, E);
        rc = sco_gather_cic(n, R, &mesh, E, Et);
        if (rc) goto done;
        const double betaC = sqrt(gammaz * gammaz - 1.0) / gammaz / SCO_C;
        for (long long i = 0; i < n; ++i) {
            Bf[3 * i + 0] = Bf[3 * i + 0] - betaC * Et[3 * i + 1];
            Bf[3 * i + 1] = Bf[3 * i + 1] + betaC * Et[3 * i + 0];
            Ef[3 * i + 0] += Et[3 * i + 0];
            Ef[3 * i + 1] += Et[3 * i + 1];
            Ef[3 * i + 2] += Et[3 * i + 2];
        }
        /* the image charge's field (:246-427) */
        const double zshift = -(2 * mesh.origin[2] + (0 + (n2 - 1) + 1) * mesh.hr[2]) * gammaz * scaleFactor;
        rc = sco_compute_potential_shifted(prm->nr, img, hr_scaled, zshift);
        if (rc) goto done;
        for (long long c = 0; c < M; ++c) img[c] *= hvol;
        for (long long c = 0; c < M; ++c) img[c] *= prm->coupling;
        sco_neg_grad_scaled(prm->nr, img, mesh.hr, gammaz, E);
        rc = sco_gather_cic(n, R, &mesh, E, Et);
        if (rc) goto done;
        for (long long i = 0; i < n; ++i) {
            Bf[3 * i + 0] = Bf[3 * i + 0] + betaC * Et[3 * i + 1];
            Bf[3 * i + 1] = Bf[3 * i + 1] - betaC * Et[3 * i + 0];
            Ef[3 * i + 0] += Et[3 * i + 0];
            Ef[3 * i + 1] += Et[3 * i + 1];
            Ef[3 * i + 2] += Et[3 * i + 2];
        }
    }
    if (dbg) {
        dbg->mesh = mesh;
        dbg->gammaz = nbins > 0 ? gam[0] : 1.0;
    }
done:
    free(gam); free(cnt); free(rho); free(img); free(E); free(Et); free(Rb);
    return rc;
}

/* ------------------------------------------------------------------------ */
/* external fields of SOLENOID elements with ASTRA 1D magnetostatic maps      */
/* (Solenoid.cpp:163-193, Astra1DMagnetoStatic.cpp:162-196) on a straight     */
/* beamline along z (element frame = lab frame shifted by ELEMEDGE), as       */
/* computeExternalFields (ParallelTTracker.cpp:614-643) and                   */
/* updateReferenceParticle (:1134-1155) apply them.                           */
/* ------------------------------------------------------------------------ */
static sco_solenoid g_sol[SCO_MAX_ELEMENTS];
static int g_nsol = 0;

int sco_set_solenoids(const sco_solenoid* s, int n) {
    if (n < 0 || n > SCO_MAX_ELEMENTS) return SCO_ERR_ARG;
    for (int k = 0; k < n; ++k) g_sol[k] = s[k];
    g_nsol = n;
    return 0;
}

/* Solenoid::apply with Astra1DMagnetoStatic::getFieldstrength: B of one
 * element at R (element frame), 0 outside [zbegin, zbegin + range). */
void sco_solenoid_field(const sco_solenoid* e, const double* R, double* B) {
    B[0] = B[1] = B[2] = 0.0;
    const double tmpR[3] = {R[0], R[1], R[2] - e->zbegin};
    if (!(tmpR[2] >= 0.0 && tmpR[2] < e->range)) return;
    const double two_pi = 2 * SCO_PI;
    const double RR2 = tmpR[0] * tmpR[0] + tmpR[1] * tmpR[1];
    const double kz = two_pi * tmpR[2] / e->period + SCO_PI;
    double ez = e->coefs[0], ezp = 0.0, ezpp = 0.0, ezppp = 0.0;
    int n = 1;
    for (int l = 1; l < e->accuracy; l++, n += 2) {
        double somefactor_base = two_pi / e->period * l;
        double somefactor = 1.0;
        double coskzl = cos(kz * l);
        double sinkzl = sin(kz * l);
        ez += (e->coefs[n] * coskzl - e->coefs[n + 1] * sinkzl);
        somefactor *= somefactor_base;
        ezp += somefactor * (-e->coefs[n] * sinkzl - e->coefs[n + 1] * coskzl);
        somefactor *= somefactor_base;
        ezpp += somefactor * (-e->coefs[n] * coskzl + e->coefs[n + 1] * sinkzl);
        somefactor *= somefactor_base;
        ezppp += somefactor * (e->coefs[n] * sinkzl + e->coefs[n + 1] * coskzl);
    }
    const double BfieldR = -ezp / 2. + ezppp / 16. * RR2;
    const double tB[3] = {BfieldR * tmpR[0], BfieldR * tmpR[1], ez - ezpp * RR2 / 4.};
    B[0] = e->scale * tB[0];
    B[1] = e->scale * tB[1];
    B[2] = e->scale * tB[2];
}

/* RFCavity::apply (RFCavity.cpp:232-249) with Astra1DDynamic::getFieldstrength
 * (Astra1DDynamic.cpp:192-229): E and B of one element at R (element frame)
 * and time t added to E, B; nothing outside [zbegin, zbegin + range). */
void sco_rfcavity_field(const sco_solenoid* e, const double* R, double t, double* E, double* B) {
    const double tmpR[3] = {R[0], R[1], R[2] - e->zbegin};
    if (!(tmpR[2] >= 0.0 && tmpR[2] < e->range)) return;
    const double two_pi = 2 * SCO_PI;
    const double RR2 = tmpR[0] * tmpR[0] + tmpR[1] * tmpR[1];
    const double kz = two_pi * tmpR[2] / e->period + SCO_PI;
    double ez = e->coefs[0], ezp = 0.0, ezpp = 0.0, ezppp = 0.0;
    int n = 1;
    for (int l = 1; l < e->accuracy; ++l, n += 2) {
        double somefactor_base = two_pi / e->period * l;
        double somefactor = 1.0;
        double coskzl = cos(kz * l);
        double sinkzl = sin(kz * l);
        ez += (e->coefs[n] * coskzl - e->coefs[n + 1] * sinkzl);
        somefactor *= somefactor_base;
        ezp += somefactor * (-e->coefs[n] * sinkzl - e->coefs[n + 1] * coskzl);
        somefactor *= somefactor_base;
        ezpp += somefactor * (-e->coefs[n] * coskzl + e->coefs[n + 1] * sinkzl);
        somefactor *= somefactor_base;
        ezppp += somefactor * (e->coefs[n] * sinkzl + e->coefs[n + 1] * coskzl);
    }
    const double f = -(ezpp + ez * e->xlrep * e->xlrep) / 16.;
    const double fp = -(ezppp + ezp * e->xlrep * e->xlrep) / 16.;
    const double EfieldR = -(ezp / 2. + fp * RR2);
    const double BfieldT = (ez / 2. + f * RR2) * e->xlrep / SCO_C;
    double tE[3] = {0.0, 0.0, 0.0}, tB[3] = {0.0, 0.0, 0.0};
    tE[0] += EfieldR * tmpR[0];
    tE[1] += EfieldR * tmpR[1];
    tE[2] += ez + 4. * f * RR2;
    tB[0] += -BfieldT * tmpR[1];
    tB[1] += BfieldT * tmpR[0];
    const double c = e->scale * cos(e->omega * t + e->phase);
    const double s = e->scale * sin(e->omega * t + e->phase);
    for (int d = 0; d < 3; ++d) {
        E[d] += c * tE[d];
        B[d] -= s * tB[d];
    }
}

/* Multipole::setNormalComponent / setSkewComponent (Multipole.cpp:106-163):
 * order n (1 = dipole): dipole and sextupole halved, the normal octupole and
 * decapole over 24, the skew octupole over 6 and decapole over 24, the
 * others as given; the dipole's stored error is its whole value. */
double sco_multipole_component(int n, int skew, double v, double verr, double* err) {
    double c, e;
    switch (n - 1) {
    case 0: c = (v + verr) / 2; e = c; break;
    case 2: c = (v + verr) / 2; e = verr / 2; break;
    case 3:
        if (skew) { c = (v + verr) / 6; e = verr / 6; }
        else { c = (v + verr) / 24; e = verr / 24; }
        break;
    case 4: c = (v + verr) / 24; e = verr / 24; break;
    default: c = (v + verr); e = verr;
    }
    if (err) *err = e;
    return c;
}

/* Multipole::computeField for one kind of components k[0..m), added to B
 * (Multipole.cpp:229-290 normal, :292-349 skew) */
static void multipole_terms(const double* k, int m, int skew, const double* R, double* B) {
    double Rn[SCO_MAX_MULTIPOLE + 1][2], fact[SCO_MAX_MULTIPOLE + 1];
    Rn[0][0] = 1.0;
    Rn[0][1] = 1.0;
    fact[0] = 1;
    for (int i = 0; i < m; ++i) {
        if (!skew) {
            if (i == 0) {
                B[1] += k[i];
            } else if (i == 1) {
                B[0] += k[i] * R[1];
                B[1] += k[i] * R[0];
            } else if (i == 2) {
                B[0] += 2 * k[i] * R[0] * R[1];
                B[1] += k[i] * (Rn[2][0] - Rn[2][1]);
            } else if (i == 3) {
                B[0] += k[i] * (3 * Rn[2][0] * Rn[1][1] - Rn[3][1]);
                B[1] += k[i] * (Rn[3][0] - 3 * Rn[1][0] * Rn[2][1]);
            } else if (i == 4) {
                B[0] += 4 * k[i] * (Rn[3][0] * Rn[1][1] - Rn[1][0] * Rn[3][1]);
                B[1] += k[i] * (Rn[4][0] - 6 * Rn[2][0] * Rn[2][1] + Rn[4][1]);
            } else {
                double sgn = 1, Bx = 0.0, By = 0.0;
                for (int j = 1; j <= (i + 1) / 2; ++j) {
                    Bx += sgn * k[i] * (Rn[i - 2 * j + 1][0] * fact[i - 2 * j + 1] * Rn[2 * j - 1][1] * fact[2 * j - 1]);
                    By += sgn * k[i] * (Rn[i - 2 * j + 2][0] * fact[i - 2 * j + 2] * Rn[2 * j - 2][1] * fact[2 * j - 2]);
                    sgn *= -1;
                }
                if ((i + 1) / 2 == i / 2) {
                    const int j = (i + 2) / 2;
                    By += sgn * k[i] * (Rn[i - 2 * j + 2][0] * fact[i - 2 * j + 2] * Rn[2 * j - 2][1] * fact[2 * j - 2]);
                }
                B[0] += Bx;
                B[1] += By;
            }
        } else {
            if (i == 0) {
                B[0] -= k[i];
            } else if (i == 1) {
                B[0] -= k[i] * R[0];
                B[1] += k[i] * R[1];
            } else if (i == 2) {
                B[0] -= k[i] * (Rn[2][0] - Rn[2][1]);
                B[1] += 2 * k[i] * R[0] * R[1];
            } else if (i == 3) {
                B[0] -= k[i] * (Rn[3][0] - 3 * Rn[1][0] * Rn[2][1]);
                B[1] += k[i] * (3 * Rn[2][0] * Rn[1][1] - Rn[3][1]);
            } else if (i == 4) {
                B[0] -= k[i] * (Rn[4][0] - 6 * Rn[2][0] * Rn[2][1] + Rn[4][1]);
                B[1] += 4 * k[i] * (Rn[3][0] * Rn[1][1] - Rn[1][0] * Rn[3][1]);
            } else {
                double sgn = 1, Bx = 0, By = 0;
                for (int j = 1; j <= (i + 1) / 2; ++j) {
                    Bx -= sgn * k[i] * (Rn[i - 2 * j + 2][0] * fact[i - 2 * j + 2] * Rn[2 * j - 2][1] * fact[2 * j - 2]);
                    By += sgn * k[i] * (Rn[i - 2 * j + 1][0] * fact[i - 2 * j + 1] * Rn[2 * j - 1][1] * fact[2 * j - 1]);
                    sgn *= -1;
                }
                if ((i + 1) / 2 == i / 2) {
                    const int j = (i + 2) / 2;
                    Bx -= sgn * k[i] * (Rn[i - 2 * j + 2][0] * fact[i - 2 * j + 2] * Rn[2 * j - 2][1] * fact[2 * j - 2]);
                }
                B[0] += Bx;
                B[1] += By;
            }
        }
        Rn[i + 1][0] = Rn[i][0] * R[0];
        Rn[i + 1][1] = Rn[i][1] * R[1];
        fact[i + 1] = fact[i] / (i + 1);
    }
}

/* Multipole::apply (:352-366): nothing outside 0 <= z <= L; nothing outside
 * the aperture (ElementBase::isInsideTransverse, ELLIPTICAL; the reference
 * also marks such a particle lost) */
void sco_multipole_field(const sco_solenoid* e, const double* R, int ref_particle, double* B) {
    if (R[2] < 0.0 || R[2] > e->range) return;
    if (!(pow(R[0] / e->aperture[0], 2) + pow(R[1] / e->aperture[1], 2) < 1.0)) return;
    const int nn = e->accuracy, ns = e->nskew;
    double k[SCO_MAX_MULTIPOLE];
    for (int i = 0; i < nn; ++i) k[i] = ref_particle ? e->coefs[i] - e->coefs[nn + i] : e->coefs[i];
    multipole_terms(k, nn, 0, R, B);
    for (int i = 0; i < ns; ++i) k[i] = ref_particle ? e->coefs[2 * nn + i] - e->coefs[2 * nn + ns + i] : e->coefs[2 * nn + i];
    multipole_terms(k, ns, 1, R, B);
}

/* bilinear interpolation of component F on a 2D map (FM2DMagnetoStatic.cpp:
 * 166-182, FM2DDynamic.cpp:195-210); absi: the magnetostatic map's abs() of
 * the floored indices; returns 0 outside the grid */
static int grid2d(const sco_solenoid* e, double RR, double z, int absi, int* i1, double* lr, double* lz) {
    int indexr = (int)floor(RR / e->hr);
    int indexz = (int)floor(z / e->hz);
    if (absi) {
        indexr = abs(indexr);
        indexz = abs(indexz);
    }
    *lr = (RR / e->hr) - indexr;
    *lz = (z / e->hz) - indexz;
    if ((indexz < 0) || (indexz + 2 > e->nz)) return 0;
    if (indexr + 2 > e->nr) return 0;
    *i1 = indexz + indexr * e->nz;
    return 1;
}
static double grid2d_at(const double* F, int index1, int nz, double leverr, double leverz) {
    const int index2 = index1 + nz;
    return (1.0 - leverz) * (1.0 - leverr) * F[index1]
         + leverz         * (1.0 - leverr) * F[index1 + 1]
         + (1.0 - leverz) * leverr         * F[index2]
         + leverz         * leverr         * F[index2 + 1];
}

void sco_solenoid2d_field(const sco_solenoid* e, const double* R, double* B) {
    B[0] = B[1] = B[2] = 0.0;
    const double tmpR[3] = {R[0], R[1], R[2] - e->zbegin};
    if (!(tmpR[2] >= 0.0 && tmpR[2] < e->range)) return;
    const double RR = sqrt(tmpR[0] * tmpR[0] + tmpR[1] * tmpR[1]);
    int i1;
    double lr, lz;
    if (!grid2d(e, RR, tmpR[2], 1, &i1, &lr, &lz)) return;
    const size_t np = (size_t)e->nz * e->nr;
    const double BfieldR = grid2d_at(e->grid + np, i1, e->nz, lr, lz);
    const double BfieldZ = grid2d_at(e->grid, i1, e->nz, lr, lz);
    double tmpB[3] = {0.0, 0.0, 0.0};
    if (RR != 0) {
        tmpB[0] += BfieldR * tmpR[0] / RR;
        tmpB[1] += BfieldR * tmpR[1] / RR;
    }
    tmpB[2] += BfieldZ;
    for (int d = 0; d < 3; ++d) B[d] += e->scale * tmpB[d];
}

void sco_rfcavity2d_field(const sco_solenoid* e, const double* R, double t, double* E, double* B) {
    const double tmpR[3] = {R[0], R[1], R[2] - e->zbegin};
    if (!(tmpR[2] >= 0.0 && tmpR[2] < e->range)) return;
    const double RR = sqrt(tmpR[0] * tmpR[0] + tmpR[1] * tmpR[1]);
    int i1;
    double lr, lz;
    if (!grid2d(e, RR, tmpR[2], 0, &i1, &lr, &lz)) return;
    const size_t np = (size_t)e->nz * e->nr;
    const double EfieldR = grid2d_at(e->grid + np, i1, e->nz, lr, lz);
    const double EfieldZ = grid2d_at(e->grid, i1, e->nz, lr, lz);
    const double BfieldT = grid2d_at(e->grid + 2 * np, i1, e->nz, lr, lz);
    double tE[3] = {0.0, 0.0, 0.0}, tB[3] = {0.0, 0.0, 0.0};
    if (RR > 1e-10) {
        tE[0] += EfieldR * tmpR[0] / RR;
        tE[1] += EfieldR * tmpR[1] / RR;
        tB[0] -= BfieldT * tmpR[1] / RR;
        tB[1] += BfieldT * tmpR[0] / RR;
    }
    tE[2] += EfieldZ;
    const double c = e->scale * cos(e->omega * t + e->phase);
    const double s = e->scale * sin(e->omega * t + e->phase);
    for (int d = 0; d < 3; ++d) {
        E[d] += c * tE[d];
        B[d] -= s * tB[d];
    }
}

/* FM3DDynamic::getFieldstrength (FM3DDynamic.cpp:242-315): the floored
 * coordinates kept as unsigned ints, the 8-term trilinear sums per component
 * in the reference's order; then RFCavity::apply's scaling (RFCavity.cpp:
 * 237-248).  No field from the last two z planes on; none (a lost particle
 * in the reference) from the last two x or y planes on. */
static unsigned idx3d(double u) {
    const double f = floor(u);
    if (!(f >= -2147483648.0 && f < 2147483647.0)) return 0xffffffffu;
    return (unsigned)(int)f;
}
void sco_rfcavity3d_field(const sco_solenoid* e, const double* R, double t, double* E, double* B) {
    const double tmpR[3] = {R[0], R[1], R[2] - e->zbegin};
    if (!(tmpR[2] >= 0.0 && tmpR[2] < e->range)) return;
    const unsigned index_x = idx3d((tmpR[0] - e->xbegin) / e->hx);
    const unsigned index_y = idx3d((tmpR[1] - e->ybegin) / e->hy);
    const unsigned index_z = idx3d(tmpR[2] / e->hz);
    if (index_z >= (unsigned)e->nz - 2u) return;
    if (index_x >= (unsigned)e->nx - 2u || index_y >= (unsigned)e->ny - 2u) return;
    const double lever_x = (tmpR[0] - e->xbegin) / e->hx - index_x;
    const double lever_y = (tmpR[1] - e->ybegin) / e->hy - index_y;
    const double lever_z = tmpR[2] / e->hz - index_z;
    const size_t deltaX = (size_t)e->ny * e->nz, deltaY = (size_t)e->nz, deltaZ = 1;
    const size_t index1 = index_x * deltaX + index_y * deltaY + index_z * deltaZ;
    const size_t np = (size_t)e->nx * deltaX;
    double tmpE[3] = {0.0, 0.0, 0.0}, tmpB[3] = {0.0, 0.0, 0.0};
    for (int c = 0; c < 6; ++c) {
        const double* F = e->grid + c * np;
        const double v = (1.0 - lever_x) * (1.0 - lever_y) * (1.0 - lever_z) * F[index1]
                       + lever_x         * (1.0 - lever_y) * (1.0 - lever_z) * F[index1 + deltaX]
                       + (1.0 - lever_x) * lever_y         * (1.0 - lever_z) * F[index1 + deltaY]
                       + lever_x         * lever_y         * (1.0 - lever_z) * F[index1 + deltaX + deltaY]
                       + (1.0 - lever_x) * (1.0 - lever_y) * lever_z         * F[index1 + deltaZ]
                       + lever_x         * (1.0 - lever_y) * lever_z         * F[index1 + deltaX + deltaZ]
                       + (1.0 - lever_x) * lever_y         * lever_z         * F[index1 + deltaY + deltaZ]
                       + lever_x         * lever_y         * lever_z         * F[index1 + deltaX + deltaY + deltaZ];
        if (c < 3)
            tmpE[c] += v;
        else
            tmpB[c - 3] += v;
    }
    const double cs = e->scale * cos(e->omega * t + e->phase);
    const double sn = e->scale * sin(e->omega * t + e->phase);
    for (int d = 0; d < 3; ++d) {
        E[d] += cs * tmpE[d];
        B[d] -= sn * tmpB[d];
    }
}

/* one element's E (RF cavities) and B at R (element frame), time t */
static void element_field(const sco_solenoid* e, const double* R, double t, int ref_particle, double* E, double* B) {
    E[0] = E[1] = E[2] = 0.0;
    if (e->kind == 1) {
        B[0] = B[1] = B[2] = 0.0;
        if (e->map3d)
            sco_rfcavity3d_field(e, R, t, E, B);
        else if (e->map2d)
            sco_rfcavity2d_field(e, R, t, E, B);
        else
            sco_rfcavity_field(e, R, t, E, B);
    } else if (e->kind == 0 && e->map2d) {
        sco_solenoid2d_field(e, R, B);
    } else if (e->kind == 2) {
        B[0] = B[1] = B[2] = 0.0;
        sco_multipole_field(e, R, ref_particle, B);
    } else {
        sco_solenoid_field(e, R, B);
    }
}

static void element_lab2local(const sco_solenoid* e, sco_trafo* t) {
    const double o[3] = {0.0, 0.0, e->edge}, q[4] = {1.0, 0.0, 0.0, 0.0};
    sco_trafo_make(t, o, q);
}

/* the particles at time t: refToLocal = misalignment * (lab2local *
   referenceToLab); E and B rotated back (localToRef.rotateTo) */
static void add_element_fields(const sco_trafo* ref_to_lab, long long n, const double* R, double t, double* Ef,
                               double* Bf) {
    for (int k = 0; k < g_nsol; ++k) {
        sco_trafo l2l, r2loc, mis;
        element_lab2local(&g_sol[k], &l2l);
        r2loc = l2l;
        sco_trafo_compose(&r2loc, ref_to_lab);
        const double o[3] = {0.0, 0.0, 0.0}, q[4] = {1.0, 0.0, 0.0, 0.0};
        sco_trafo_make(&mis, o, q);
        sco_trafo_compose(&mis, &r2loc);
        r2loc = mis;
        sco_trafo loc2r = r2loc;
        sco_trafo_invert(&loc2r);
        SCO_PAR
        for (long long i = 0; i < n; ++i) {
            double loc[3], El[3], Bl[3], Er[3], Br[3];
            trafo_transform_to(&r2loc, R + 3 * i, loc);
            element_field(&g_sol[k], loc, t, 0, El, Bl);
            trafo_rotate_to(&loc2r, Bl, Br);
            Bf[3 * i + 0] += Br[0];
            Bf[3 * i + 1] += Br[1];
            Bf[3 * i + 2] += Br[2];
            if (g_sol[k].kind == 1) {
                trafo_rotate_to(&loc2r, El, Er);
                Ef[3 * i + 0] += Er[0];
                Ef[3 * i + 1] += Er[1];
                Ef[3 * i + 2] += Er[2];
            }
        }
    }
}

/* the reference particle at time t: refToLocal = lab2local * referenceToLab,
   E and B rotated from */
static void add_element_fields_ref(const sco_trafo* ref_to_lab, const double* R, double t, double* Ef, double* Bf) {
    for (int k = 0; k < g_nsol; ++k) {
        sco_trafo r2loc;
        element_lab2local(&g_sol[k], &r2loc);
        sco_trafo_compose(&r2loc, ref_to_lab);
        double loc[3], El[3], Bl[3];
        trafo_transform_to(&r2loc, R, loc);
        element_field(&g_sol[k], loc, t, 1, El, Bl);
        const double* M = r2loc.M;
        Bf[0] += M[0] * Bl[0] + M[3] * Bl[1] + M[6] * Bl[2];
        Bf[1] += M[1] * Bl[0] + M[4] * Bl[1] + M[7] * Bl[2];
        Bf[2] += M[2] * Bl[0] + M[5] * Bl[1] + M[8] * Bl[2];
        if (g_sol[k].kind == 1) {
            Ef[0] += M[0] * El[0] + M[3] * El[1] + M[6] * El[2];
            Ef[1] += M[1] * El[0] + M[4] * El[1] + M[7] * El[2];
            Ef[2] += M[2] * El[0] + M[5] * El[1] + M[8] * El[2];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* one ParallelTTracker step (ParallelTTracker.cpp:343-365)                   */
/* bins == NULL: computeSelfFields(); else the energy-bin loop (:567-578).    */
/* ------------------------------------------------------------------------ */
static int tracker_step(sco_tracker* tr, long long n, double* R, double* P, double* Ef, double* Bf,
                        const sco_bins* bins, sco_debug* dbg) {
    const sco_params* prm = &tr->prm;
    const double dT = prm->dT;
    /* timeIntegration1 -> pushParticles (:434-447, .h:448-455) */
    sco_push(n, R, P, dT);
    /* Ef = Bf = 0 (:347-348) */
    memset(Ef, 0, 3 * n * sizeof(double));
    memset(Bf, 0, 3 * n * sizeof(double));
    /* computeSpaceChargeFields (:546-592) */
    double m27[27];
    sco_moments(n, R, P, m27);
    const double N = (double)n;
    double pmean[3] = {m27[1] / N, m27[3] / N, m27[5] / N};
    double zhat[3] = {0.0, 0.0, 1.0}, q[4];
    if (sco_get_quaternion(pmean, zhat, q)) return SCO_ERR_FRAME;
    double qc[4] = {q[0], -q[1], -q[2], -q[3]};
    double org[3] = {0.0, 0.0, tr->path_length};
    sco_trafo b2r, r2b;
    sco_trafo_make(&b2r, org, qc);
    r2b = b2r;
    sco_trafo_invert(&r2b);
    SCO_PAR
    for (long long i = 0; i < n; ++i) {
        double v[3];
        trafo_transform_to(&r2b, R + 3 * i, v);
        R[3 * i] = v[0]; R[3 * i + 1] = v[1]; R[3 * i + 2] = v[2];
    }
    int rc;
    if (bins)
        rc = sco_compute_self_fields_binned(prm, tr->Q, n, R, P, bins->bin, bins->nbins, bins->last_emitted, Ef, Bf,
                                            NULL, dbg);
    else
        rc = sco_compute_self_fields(prm, &tr->Q, n, R, P, Ef, Bf, dbg);
    if (rc) return rc;
    SCO_PAR
    for (long long i = 0; i < n; ++i) {
        double v[3];
        trafo_transform_to(&b2r, R + 3 * i, v);
        R[3 * i] = v[0]; R[3 * i + 1] = v[1]; R[3 * i + 2] = v[2];
        trafo_rotate_to(&b2r, Ef + 3 * i, v);
        Ef[3 * i] = v[0]; Ef[3 * i + 1] = v[1]; Ef[3 * i + 2] = v[2];
        trafo_rotate_to(&b2r, Bf + 3 * i, v);
        Bf[3 * i] = v[0]; Bf[3 * i + 1] = v[1]; Bf[3 * i + 2] = v[2];
    }
    if (dbg) {
        memcpy(dbg->rot_beam_to_ref, b2r.M, sizeof(b2r.M));
        dbg->pmean[0] = pmean[0]; dbg->pmean[1] = pmean[1]; dbg->pmean[2] = pmean[2];
    }
    /* computeExternalFields (:356): a uniform solenoid field along z */
    if (prm->bz_ext != 0.0) {
        SCO_PAR
        for (long long i = 0; i < n; ++i) Bf[3 * i + 2] += prm->bz_ext;
    }
    /* the particles' field time: getT() + 0.5 dt (:628) */
    add_element_fields(&tr->ref_to_lab, n, R, tr->t + 0.5 * dT, Ef, Bf);
    if (dbg && dbg->Ef) memcpy(dbg->Ef, Ef, 3 * n * sizeof(double));
    if (dbg && dbg->Bf) memcpy(dbg->Bf, Bf, 3 * n * sizeof(double));
    /* timeIntegration2: kick + push (:450-491) */
    sco_kick(n, P, Ef, Bf, dT, prm->mass, prm->charge);
    sco_push(n, R, P, dT);
    /* t += dT; updateRefToLabCSTrafo (:360-365, :1123-1212) */
    tr->t += dT;
    if (tr->t > 0.0) {
        const double dt = tr->t < dT ? tr->t : dT;
        const double scaleFactor = SCO_C * dt;
        double* rr = tr->ref_R;
        double* rp = tr->ref_P;
        double eref[3] = {0.0, 0.0, 0.0}, bref[3] = {0.0, 0.0, 0.0};
        rr[0] /= scaleFactor; rr[1] /= scaleFactor; rr[2] /= scaleFactor;
        { double g = sqrt(1.0 + dot3(rp, rp)); rr[0] += 0.5 * rp[0] / g; rr[1] += 0.5 * rp[1] / g; rr[2] += 0.5 * rp[2] / g; }
        rr[0] *= scaleFactor; rr[1] *= scaleFactor; rr[2] *= scaleFactor;
        /* the reference particle's field time: getT() - 0.5 dt (:1149) */
        add_element_fields_ref(&tr->ref_to_lab, rr, tr->t - 0.5 * dt, eref, bref);
        if (prm->bz_ext != 0.0) bref[2] += prm->bz_ext;
        kick_one(rp, eref, bref, dt, prm->mass, prm->charge);
        rr[0] /= scaleFactor; rr[1] /= scaleFactor; rr[2] /= scaleFactor;
        { double g = sqrt(1.0 + dot3(rp, rp)); rr[0] += 0.5 * rp[0] / g; rr[1] += 0.5 * rp[1] / g; rr[2] += 0.5 * rp[2] / g; }
        rr[0] *= scaleFactor; rr[1] *= scaleFactor; rr[2] *= scaleFactor;
        tr->path_length += sqrt(dot3(rr, rr));
        double qu[4];
        if (sco_get_quaternion(rp, zhat, qu)) return SCO_ERR_FRAME;
        sco_trafo upd;
        sco_trafo_make(&upd, rr, qu);
        double v[3];
        trafo_transform_to(&upd, rr, v);
        rr[0] = v[0]; rr[1] = v[1]; rr[2] = v[2];
        trafo_rotate_to(&upd, rp, v);
        rp[0] = v[0]; rp[1] = v[1]; rp[2] = v[2];
        SCO_PAR
        for (long long i = 0; i < n; ++i) {
            double w[3];
            trafo_transform_to(&upd, R + 3 * i, w);
            R[3 * i] = w[0]; R[3 * i + 1] = w[1]; R[3 * i + 2] = w[2];
            trafo_rotate_to(&upd, P + 3 * i, w);
            P[3 * i] = w[0]; P[3 * i + 1] = w[1]; P[3 * i + 2] = w[2];
        }
        sco_trafo inv = upd;
        sco_trafo_invert(&inv);
        sco_trafo_compose(&tr->ref_to_lab, &inv);
        if (dbg) memcpy(dbg->update_origin, upd.origin, sizeof(upd.origin));
    }
    tr->step += 1;
    return 0;
}

int sco_tracker_init(sco_tracker* tr, const sco_params* prm, double Q) {
    memset(tr, 0, sizeof(*tr));
    tr->prm = *prm;
    tr->Q = Q;
    tr->ref_P[2] = prm->ref_pz;
    double o[3] = {0.0, 0.0, 0.0}, q[4] = {1.0, 0.0, 0.0, 0.0};
    sco_trafo_make(&tr->ref_to_lab, o, q);
    return 0;
}

static int track_impl(sco_tracker* tr, long long n, double* R, double* P, const sco_bins* bins, int nsteps,
                      sco_debug* dbg) {
    if (n <= 0) return SCO_ERR_ARG;
    double* Ef = (double*)malloc(3 * n * sizeof(double));
    double* Bf = (double*)malloc(3 * n * sizeof(double));
    if (!Ef || !Bf) { free(Ef); free(Bf); return SCO_ERR_OOM; }
    int rc = 0;
    for (int s = 0; s < nsteps && rc == 0; ++s)
        rc = tracker_step(tr, n, R, P, Ef, Bf, bins, (s == nsteps - 1) ? dbg : NULL);
    free(Ef);
    free(Bf);
    return rc;
}

int sco_track(sco_tracker* tr, long long n, double* R, double* P, int nsteps, sco_debug* dbg) {
    return track_impl(tr, n, R, P, NULL, nsteps, dbg);
}

/* the step loop with energy bins: bin[i] in [0, nbins) per particle (the
 * bins travel with the particles; the loop covers bins below
 * min(last_emitted, nbins)) */
int sco_track_binned(sco_tracker* tr, long long n, double* R, double* P, const int* bin, int nbins,
                     int last_emitted, int nsteps, sco_debug* dbg) {
    if (!bin || nbins <= 0) return SCO_ERR_ARG;
    sco_bins b = {bin, nbins, last_emitted};
    return track_impl(tr, n, R, P, &b, nsteps, dbg);
}

int sco_sizeof_tracker(void) { return (int)sizeof(sco_tracker); }
int sco_sizeof_debug(void) { return (int)sizeof(sco_debug); }
int sco_sizeof_beam_params(void) { return (int)sizeof(sco_beam_params); }
