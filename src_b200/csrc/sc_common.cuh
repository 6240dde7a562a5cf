// sc_common.cuh -- types and scalar math shared by the host and the device.
//
// The scalar frame arithmetic below (quaternions, coordinate-system
// transformations, the Boris pusher) follows OPAL's expressions operand for
// operand so that, compiled without fused multiply-add contraction, the
// device computes the same doubles as the reference's CPU code:
//   Quaternion.cpp:34-150, CoordinateSystemTrafo.{h:77-85,cpp:18-43},
//   BorisPusher.h:56-124, PartBunchBase.hpp:468-513.
// Only +, -, *, / and sqrt appear; all are correctly rounded on both sides.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#define SC_HD __host__ __device__ __forceinline__
// once-per-step scalar work run by one thread of a last block: kept out of line
// so that it does not raise the register budget of the particle loops
#define SC_HD_COLD inline __host__ __device__ __noinline__

namespace sc {

constexpr double kC = 299792458.0;          // Physics.h:52
constexpr double kPi = 3.14159265358979323846;  // Physics.h:31

// status codes (mirrored by include/scgpu.h)
enum : int {
    kOk = 0,
    kErrArg = -1,
    kErrOom = -2,
    kErrMesh = -3,
    kErrGuard = -4,
    kErrFrame = -5,
    kErrCuda = -6,
    kErrState = -7,
    kErrUnsupported = -8,
};

// device-side error bits (StepState::err)
enum : int {
    kFlagMesh = 1,
    kFlagGuard = 2,
    kFlagFrame = 4,
    kFlagSort = 8,  // a sort position fell outside [0, N): inconsistent histogram
    kFlagBin = 16,  // an energy bin outside [0, nbins)
    kFlagCopy = 32, // a bulk copy into shared memory did not complete in time
};

struct Trafo {
    double origin[3];
    double quat[4];
    double M[9];  // row-major
};

// Device-resident state of one bunch: the ParallelTTracker members that the
// step loop updates, and the per-step scalars that one kernel derives and
// later kernels read.  Kernels read it through a pointer so that a captured
// CUDA graph replays correctly for any number of steps.
struct StepState {
    // tracker state
    double t;
    double path_length;
    double ref_R[3];
    double ref_P[3];
    Trafo ref_to_lab;
    double Q;  // macro-particle charge after the Q*=dt ... Q/=dt round trip
    long long step;
    unsigned int gen;  // deposit generation stamp (never 0 once a step ran)
    int err;
    // reductions of the particle state at the end of the previous step
    double psum[3];
    double moments[27];
    double gsum;
    // per-step scalars
    Trafo r2b;  // reference -> beam frame (inverse of b2r)
    Trafo b2r;  // beam -> reference frame
    double bmin[3], bmax[3];
    double mesh_rmin[3], mesh_rmax[3];
    double hr[3], origin[3];
    double rhr[3];  // RN(1 / hr)
    double gammaz;
    double hr_scaled[3];
    double tmp2;   // 1/hx * 1/hy * 1/hz_scaled
    double hvol;   // hx * hy * hz_scaled
    double betaC;  // sqrt(gz^2-1)/gz/c
    double qdt;    // Q * dt (the scattered charge)
    Trafo upd;     // reference-particle update of this step
    Trafo ref_to_lab_step;  // ref -> lab at the start of the step (the external fields' frame)
    double t_step;          // t at the start of the step (the particles' field time is t_step + dT / 2)
    // energy bins / image charge
    double zshift;      // z shift of the image's Green's function (PartBunch.cpp:249)
    long long bin_count;  // particles in the bin (per-bin copies)
    int binned;         // the energy-bin loop is on: Q is restored after the scatter (ParallelTTracker.cpp:576)
    int pad_;
    // sharded bunch: this rank's partial results, combined over the ranks
    // between kernels (bounds by min; exact sums as 32-bit chunks of the
    // 128-bit fixed point, summed as 64-bit integers)
    double bnd6[6];                 // min x, y, z and -max x, y, z
    unsigned long long xlimbs[28 * 4];
};

// A beamline element with a 1D field map in ASTRA format on a straight
// beamline along z (element frame = lab frame shifted by ELEMEDGE):
//  * SOLENOID with a magnetostatic map (Solenoid.cpp:163-215;
//    Astra1DMagnetoStatic.cpp:162-196), scaled by KS [T];
//  * RFCAVITY with a dynamic (standing-wave) map (RFCavity.cpp:232-270;
//    Astra1DDynamic.cpp:162-229), scaled by VOLT [MV/m], oscillating as
//    cos(omega t + LAG) (E) and sin(omega t + LAG) (B).
constexpr int kMaxSolCoefs = 255;  // 2 accuracy - 1, accuracy <= 128
constexpr int kMaxElements = 8;
constexpr int kMaxMultipoleOrder = 20;  // components per kind (normal, skew) of a MULTIPOLE
enum : int { kElemSolenoid = 0, kElemRfCavity = 1, kElemMultipole = 2 };
struct MapElem {
    double edge;    // ELEMEDGE: the element origin on the lab z axis [m]
    double scale;   // KS [T] or VOLT [MV/m] (the map is normalised to 1 T, or to 1 MV/m in V/m)
    double zbegin;  // startField: the map's first z (element frame)
    double range;   // zend - zbegin: the field region (the element's length)
    double period;  // 2 N (zend - zbegin) / (N - 1): the Fourier period
    int accuracy;   // harmonics 0 .. accuracy - 1; MULTIPOLE: normal components
    int kind;       // kElemSolenoid, kElemRfCavity or kElemMultipole
    double omega;   // RF: angular frequency [rad/s]
    double phase;   // RF: LAG [rad]
    double xlrep;   // RF: the map's angular frequency / c [1/m]
    int nskew;      // MULTIPOLE: skew components
    int map2d;      // SOLENOID / RFCAVITY: 1 for a 2D (r, z) grid map in place of the 1D series
    double aperture[2];  // MULTIPOLE: semi-axes of the elliptical aperture [m]
    // 2D map: grid points along z and r, spacings, and the device grid
    // (Bz, Br or Ez, Er, Bt, each nz nr values, z fastest)
    int nz, nr;
    double hz, hr;
    const double* grid;
    // 3D map of an RFCAVITY (FM3DDynamic): 1, the grid points along x and y
    // (nz above), spacings and the map's first x and y; the grid holds Ex, Ey,
    // Ez [V/m], Bx, By, Bz [T], each nx ny nz values, (x i, y j, z k) at
    // (i ny + j) nz + k
    int map3d, nx, ny, pad3_;
    double hx, hy, xbegin, ybegin;
    // map: Fourier coefficients; MULTIPOLE: normal components, their errors,
    // skew components, their errors (accuracy, accuracy, nskew, nskew values)
    double coefs[kMaxSolCoefs];
};

struct BunchConst {
    int n[3];       // mesh cells per axis (MX, MY, MT)
    int key_bits;
    long long N;    // particles (of this rank when the bunch is sharded)
    long long Ntot; // particles of the whole bunch (the N of the means)
    int sharded;    // 1: bounds and particle sums are combined over ranks between kernels
    int pz;         // 1: DC beam (periodic z: the period's mesh, the periodic particle boundary)
    double dT;
    double mass;    // eV
    double charge;  // e
    double coupling;
    double bz_ext;
    double dh;
    double period;  // DC beam: period length along z [m] (periodLength_m, c / beam frequency)
    // per-bunch constants of the pusher, evaluated in the reference's order
    double s_cdt;   // c * dT                      (PartBunchBase.hpp:481)
    double rs_cdt;  // RN(1 / (c * dT))
    double ke;      // 0.5 * dT * charge * c / mass (BorisPusher.h:88)
    double ktn;     // 0.5 * dT * charge * c * c    (BorisPusher.h:99, numerator)
    // beamline elements with external fields (device table), none when nsol == 0
    const MapElem* sol;
    int nsol;
    int pad2_;
};

// fill the derived pusher constants of bc (host side)
inline void bunch_constants(BunchConst& bc) {
    bc.s_cdt = kC * bc.dT;
    bc.rs_cdt = 1.0 / bc.s_cdt;
    bc.ke = 0.5 * bc.dT * bc.charge * kC / bc.mass;
    bc.ktn = 0.5 * bc.dT * bc.charge * kC * kC;
}

// ---------------------------------------------------------------- vectors
SC_HD double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
SC_HD void cross3(const double* a, const double* b, double* r) {
    double r0 = a[1] * b[2] - a[2] * b[1];
    double r1 = a[2] * b[0] - a[0] * b[2];
    double r2 = a[0] * b[1] - a[1] * b[0];
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
}
SC_HD void matvec(const double* M, const double* v, double* r) {
    double r0 = M[0] * v[0] + M[1] * v[1] + M[2] * v[2];
    double r1 = M[3] * v[0] + M[4] * v[1] + M[5] * v[2];
    double r2 = M[6] * v[0] + M[7] * v[1] + M[8] * v[2];
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
}

// ---------------------------------------------------------------- quaternions
SC_HD void quat_mul(const double* a, const double* b, double* r) {
    double ai[3] = {a[1], a[2], a[3]}, bi[3] = {b[1], b[2], b[3]}, c[3];
    cross3(ai, bi, c);
    double r0 = a[0] * b[0] - dot3(ai, bi);
    double r1 = a[0] * bi[0] + b[0] * ai[0] + c[0];
    double r2 = a[0] * bi[1] + b[0] * ai[1] + c[1];
    double r3 = a[0] * bi[2] + b[0] * ai[2] + c[2];
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
    r[3] = r3;
}
SC_HD void quat_normalize(double* q) {
    double len = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    q[0] /= len;
    q[1] /= len;
    q[2] /= len;
    q[3] /= len;
}
SC_HD void quat_rotate(const double* q, const double* v, double* r) {
    double qv[4] = {0.0, v[0], v[1], v[2]};
    double qc[4] = {q[0], -q[1], -q[2], -q[3]};
    double t[4], u[4];
    quat_mul(qv, qc, t);
    quat_mul(q, t, u);
    r[0] = u[1];
    r[1] = u[2];
    r[2] = u[3];
}
SC_HD void quat_rotmat(const double* qin, double* M) {
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
// getQuaternion(u, ref); false for anti-parallel or null input.
SC_HD bool get_quaternion(const double* uin, const double* refin, double* q) {
    const double tol = 1e-12;
    double u[3] = {uin[0], uin[1], uin[2]}, ref[3] = {refin[0], refin[1], refin[2]};
    double lu = sqrt(dot3(u, u)), lr = sqrt(dot3(ref, ref));
    if (!(lu >= 1e-12) || !(lr >= 1e-12)) return false;
    u[0] /= lu;
    u[1] /= lu;
    u[2] /= lu;
    ref[0] /= lr;
    ref[1] /= lr;
    ref[2] /= lr;
    double axis[3];
    cross3(u, ref, axis);
    double normAxis = sqrt(dot3(axis, axis));
    if (normAxis < tol) {
        double d = dot3(u, ref) - 1.0;
        if ((d < 0 ? -d : d) < tol) {
            q[0] = 1.0;
            q[1] = q[2] = q[3] = 0.0;
            return true;
        }
        return false;
    }
    axis[0] /= normAxis;
    axis[1] /= normAxis;
    axis[2] /= normAxis;
    double cosAngle = sqrt(0.5 * (1 + dot3(u, ref)));
    double sinAngle = sqrt(1 - cosAngle * cosAngle);
    q[0] = cosAngle;
    q[1] = sinAngle * axis[0];
    q[2] = sinAngle * axis[1];
    q[3] = sinAngle * axis[2];
    return true;
}

// ---------------------------------------------------------------- trafos
SC_HD void trafo_make(Trafo& t, const double* origin, const double* quat) {
    for (int i = 0; i < 3; ++i) t.origin[i] = origin[i];
    for (int i = 0; i < 4; ++i) t.quat[i] = quat[i];
    quat_rotmat(t.quat, t.M);
}
SC_HD void trafo_invert(Trafo& t) {
    double r[3];
    quat_rotate(t.quat, t.origin, r);
    t.origin[0] = -r[0];
    t.origin[1] = -r[1];
    t.origin[2] = -r[2];
    t.quat[1] = -t.quat[1];
    t.quat[2] = -t.quat[2];
    t.quat[3] = -t.quat[3];
    double M[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) M[i * 3 + j] = t.M[j * 3 + i];
    for (int i = 0; i < 9; ++i) t.M[i] = M[i];
}
SC_HD void trafo_compose(Trafo& t, const Trafo& right) {
    double rc[4] = {right.quat[0], -right.quat[1], -right.quat[2], -right.quat[3]};
    double r[3];
    quat_rotate(rc, t.origin, r);
    t.origin[0] = r[0] + right.origin[0];
    t.origin[1] = r[1] + right.origin[1];
    t.origin[2] = r[2] + right.origin[2];
    double q[4];
    quat_mul(t.quat, right.quat, q);
    for (int i = 0; i < 4; ++i) t.quat[i] = q[i];
    quat_normalize(t.quat);
    quat_rotmat(t.quat, t.M);
}
SC_HD void trafo_transform_to(const Trafo& t, const double* r, double* out) {
    double d[3] = {r[0] - t.origin[0], r[1] - t.origin[1], r[2] - t.origin[2]};
    matvec(t.M, d, out);
}
SC_HD void trafo_rotate_to(const Trafo& t, const double* r, double* out) { matvec(t.M, r, out); }
// the inverse rotation (the rotation matrix of the inverted trafo is M^T exactly)
SC_HD void trafo_rotate_from(const Trafo& t, const double* r, double* out) {
    const double* M = t.M;
    out[0] = M[0] * r[0] + M[3] * r[1] + M[6] * r[2];
    out[1] = M[1] * r[0] + M[4] * r[1] + M[7] * r[2];
    out[2] = M[2] * r[0] + M[5] * r[1] + M[8] * r[2];
}

// ---------------------------------------------------------------- external fields
// The Fourier series of a map's on-axis field and its first three z
// derivatives at tz = z - zbegin (the loops of Astra1DMagnetoStatic.cpp:
// 170-189 and Astra1DDynamic.cpp:199-216, one expression order).
SC_HD void map_series(const MapElem& e, double tz, double& ez, double& ezp, double& ezpp, double& ezppp) {
    const double two_pi = 2 * kPi;
    const double kz = two_pi * tz / e.period + kPi;
    ez = e.coefs[0], ezp = 0.0, ezpp = 0.0, ezppp = 0.0;
    int n = 1;
    for (int l = 1; l < e.accuracy; l++, n += 2) {
        const double base = two_pi / e.period * l;
        double f = 1.0;
        const double c = cos(kz * l), s = sin(kz * l);
        ez += (e.coefs[n] * c - e.coefs[n + 1] * s);
        f *= base;
        ezp += f * (-e.coefs[n] * s - e.coefs[n + 1] * c);
        f *= base;
        ezpp += f * (-e.coefs[n] * c + e.coefs[n + 1] * s);
        f *= base;
        ezppp += f * (e.coefs[n] * s + e.coefs[n + 1] * c);
    }
}

// Astra1DMagnetoStatic::getFieldstrength expanded off axis, for R in the
// element frame; Solenoid::apply (Solenoid.cpp:167-179): only inside
// [zbegin, zbegin + range), scaled by KS.
SC_HD void solenoid_field(const MapElem& e, const double* R, double* B) {
    const double tz = R[2] - e.zbegin;
    if (!(tz >= 0.0 && tz < e.range)) return;
    const double RR2 = R[0] * R[0] + R[1] * R[1];
    double ez, ezp, ezpp, ezppp;
    map_series(e, tz, ez, ezp, ezpp, ezppp);
    const double BfieldR = -ezp / 2. + ezppp / 16. * RR2;
    const double tB[3] = {BfieldR * R[0], BfieldR * R[1], ez - ezpp * RR2 / 4.};
    B[0] = e.scale * tB[0];
    B[1] = e.scale * tB[1];
    B[2] = e.scale * tB[2];
}

// Astra1DDynamic::getFieldstrength (:192-229): the standing-wave field of the
// on-axis E_z expanded off axis with the wave number xlrep, and
// RFCavity::apply (:232-249): inside [zbegin, zbegin + range) at time t,
// E += VOLT cos(omega t + LAG) E_map, B -= VOLT sin(omega t + LAG) B_map.
SC_HD void rfcavity_field(const MapElem& e, const double* R, double t, double* E, double* B) {
    const double tz = R[2] - e.zbegin;
    if (!(tz >= 0.0 && tz < e.range)) return;
    const double RR2 = R[0] * R[0] + R[1] * R[1];
    double ez, ezp, ezpp, ezppp;
    map_series(e, tz, ez, ezp, ezpp, ezppp);
    const double f = -(ezpp + ez * e.xlrep * e.xlrep) / 16.;
    const double fp = -(ezppp + ezp * e.xlrep * e.xlrep) / 16.;
    const double EfieldR = -(ezp / 2. + fp * RR2);
    const double BfieldT = (ez / 2. + f * RR2) * e.xlrep / kC;
    const double tE[3] = {EfieldR * R[0], EfieldR * R[1], ez + 4. * f * RR2};
    const double tB[3] = {-BfieldT * R[1], BfieldT * R[0], 0.0};
    const double arg = e.omega * t + e.phase;
    const double ce = e.scale * cos(arg), sb = e.scale * sin(arg);
    E[0] += ce * tE[0];
    E[1] += ce * tE[1];
    E[2] += ce * tE[2];
    B[0] -= sb * tB[0];
    B[1] -= sb * tB[1];
    B[2] -= sb * tB[2];
}

// Bilinear interpolation on a 2D (r, z) map at distance RR from the axis and
// height z above the map's start (FM2DMagnetoStatic.cpp:170-186,
// FM2DDynamic.cpp:192-212): false outside the grid.  ABSI: the magnetostatic
// map takes the absolute value of the floored indices.
template <bool ABSI>
SC_HD bool grid2d_cell(const MapElem& e, double RR, double z, int& i1, double& lr, double& lz) {
    int ir = (int)floor(RR / e.hr);
    int iz = (int)floor(z / e.hz);
    if (ABSI) {
        ir = ir < 0 ? -ir : ir;
        iz = iz < 0 ? -iz : iz;
    }
    lr = ABSI ? (RR / e.hr) - ir : RR / e.hr - ir;
    lz = ABSI ? (z / e.hz) - iz : z / e.hz - iz;
    if (iz < 0 || iz + 2 > e.nz) return false;
    if (ir + 2 > e.nr) return false;  // out of the map radially: the reference loses the particle
    i1 = iz + ir * e.nz;
    return true;
}
SC_HD double grid2d_value(const double* F, int i1, int nz, double lr, double lz) {
    const int i2 = i1 + nz;
    return (1.0 - lz) * (1.0 - lr) * F[i1] + lz * (1.0 - lr) * F[i1 + 1] + (1.0 - lz) * lr * F[i2] + lz * lr * F[i2 + 1];
}

// FM2DMagnetoStatic::getFieldstrength and Solenoid::apply: B = KS (Br x/r,
// Br y/r, Bz) inside [zbegin, zbegin + range).
SC_HD void solenoid2d_field(const MapElem& e, const double* R, double* B) {
    const double tz = R[2] - e.zbegin;
    if (!(tz >= 0.0 && tz < e.range)) return;
    const double RR = sqrt(R[0] * R[0] + R[1] * R[1]);
    int i1;
    double lr, lz;
    if (!grid2d_cell<true>(e, RR, tz, i1, lr, lz)) return;
    const size_t np = (size_t)e.nz * e.nr;
    const double BfieldR = grid2d_value(e.grid + np, i1, e.nz, lr, lz);
    const double BfieldZ = grid2d_value(e.grid, i1, e.nz, lr, lz);
    double tB[3] = {0.0, 0.0, 0.0};
    if (RR != 0) {
        tB[0] += BfieldR * R[0] / RR;
        tB[1] += BfieldR * R[1] / RR;
    }
    tB[2] += BfieldZ;
    B[0] += e.scale * tB[0];
    B[1] += e.scale * tB[1];
    B[2] += e.scale * tB[2];
}

// FM2DDynamic::getFieldstrength and RFCavity::apply: E += VOLT cos(omega t +
// LAG) (Er x/r, Er y/r, Ez), B -= VOLT sin(omega t + LAG) (-Bt y/r, Bt x/r, 0).
SC_HD void rfcavity2d_field(const MapElem& e, const double* R, double t, double* E, double* B) {
    const double tz = R[2] - e.zbegin;
    if (!(tz >= 0.0 && tz < e.range)) return;
    const double RR = sqrt(R[0] * R[0] + R[1] * R[1]);
    int i1;
    double lr, lz;
    if (!grid2d_cell<false>(e, RR, tz, i1, lr, lz)) return;
    const size_t np = (size_t)e.nz * e.nr;
    const double EfieldR = grid2d_value(e.grid + np, i1, e.nz, lr, lz);
    const double EfieldZ = grid2d_value(e.grid, i1, e.nz, lr, lz);
    const double BfieldT = grid2d_value(e.grid + 2 * np, i1, e.nz, lr, lz);
    double tE[3] = {0.0, 0.0, 0.0}, tB[3] = {0.0, 0.0, 0.0};
    if (RR > 1e-10) {
        tE[0] += EfieldR * R[0] / RR;
        tE[1] += EfieldR * R[1] / RR;
        tB[0] -= BfieldT * R[1] / RR;
        tB[1] += BfieldT * R[0] / RR;
    }
    tE[2] += EfieldZ;
    const double arg = e.omega * t + e.phase;
    const double ce = e.scale * cos(arg), sb = e.scale * sin(arg);
    E[0] += ce * tE[0];
    E[1] += ce * tE[1];
    E[2] += ce * tE[2];
    B[0] -= sb * tB[0];
    B[1] -= sb * tB[1];
    B[2] -= sb * tB[2];
}

// The floored grid coordinate as the reference's unsigned index
// (static_cast<int>(floor(u)) stored in an unsigned int): a point before the
// grid's start becomes a huge index, which the range checks reject.
SC_HD unsigned grid3d_index(double u) {
    const double f = floor(u);
    if (!(f >= -2147483648.0 && f < 2147483647.0)) return 0xffffffffu;
    return (unsigned)(int)f;
}
// FM3DDynamic's trilinear interpolation of one component, its terms in the
// reference's order (FM3DDynamic.cpp:262-270; x steps by dX, y by dY, z by 1)
SC_HD double grid3d_value(const double* F, size_t i1, size_t dX, size_t dY, double lx, double ly, double lz) {
    return (1.0 - lx) * (1.0 - ly) * (1.0 - lz) * F[i1] + lx * (1.0 - ly) * (1.0 - lz) * F[i1 + dX] +
           (1.0 - lx) * ly * (1.0 - lz) * F[i1 + dY] + lx * ly * (1.0 - lz) * F[i1 + dX + dY] +
           (1.0 - lx) * (1.0 - ly) * lz * F[i1 + 1] + lx * (1.0 - ly) * lz * F[i1 + dX + 1] +
           (1.0 - lx) * ly * lz * F[i1 + dY + 1] + lx * ly * lz * F[i1 + dX + dY + 1];
}

// FM3DDynamic::getFieldstrength (FM3DDynamic.cpp:242-315) with RFCavity::apply
// (RFCavity.cpp:232-250): E += VOLT cos(omega t + LAG) E_map and B -= VOLT
// sin(omega t + LAG) B_map, the map field interpolated at (x, y, z - zbegin)
// inside [zbegin, zbegin + range).  No field from the last two z planes on;
// none from the last two x or y planes on either (there the reference loses
// the particle).
SC_HD void rfcavity3d_field(const MapElem& e, const double* R, double t, double* E, double* B) {
    const double tz = R[2] - e.zbegin;
    if (!(tz >= 0.0 && tz < e.range)) return;
    const double ux = (R[0] - e.xbegin) / e.hx, uy = (R[1] - e.ybegin) / e.hy, uz = tz / e.hz;
    const unsigned ix = grid3d_index(ux), iy = grid3d_index(uy), iz = grid3d_index(uz);
    if (iz >= (unsigned)e.nz - 2u) return;
    if (ix >= (unsigned)e.nx - 2u || iy >= (unsigned)e.ny - 2u) return;
    const double lx = ux - ix, ly = uy - iy, lz = uz - iz;
    const size_t dX = (size_t)e.ny * e.nz, dY = (size_t)e.nz;
    const size_t i1 = ix * dX + iy * dY + iz, np = (size_t)e.nx * dX;
    double v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] = grid3d_value(e.grid + c * np, i1, dX, dY, lx, ly, lz);
    const double arg = e.omega * t + e.phase;
    const double ce = e.scale * cos(arg), sb = e.scale * sin(arg);
    E[0] += ce * v[0];
    E[1] += ce * v[1];
    E[2] += ce * v[2];
    B[0] -= sb * v[3];
    B[1] -= sb * v[4];
    B[2] -= sb * v[5];
}

// Multipole::computeField (Multipole.cpp:229-349): the normal components
// c[0..nn), then the skew components s[0..ns), each order's term added to
// B_x, B_y in the reference's expression order (special forms for the
// dipole .. decapole, the general series with the inverse factorials beyond).
SC_HD void multipole_terms(const double* c, int nn, bool skew, const double* R, double* B) {
    double Rn0[kMaxMultipoleOrder + 1], Rn1[kMaxMultipoleOrder + 1], fact[kMaxMultipoleOrder + 1];
    Rn0[0] = 1.0;
    Rn1[0] = 1.0;
    fact[0] = 1;
    for (int i = 0; i < nn; ++i) {
        const double k = c[i];
        if (!skew) {
            switch (i) {
                case 0:
                    B[1] += k;
                    break;
                case 1:
                    B[0] += k * R[1];
                    B[1] += k * R[0];
                    break;
                case 2:
                    B[0] += 2 * k * R[0] * R[1];
                    B[1] += k * (Rn0[2] - Rn1[2]);
                    break;
                case 3:
                    B[0] += k * (3 * Rn0[2] * Rn1[1] - Rn1[3]);
                    B[1] += k * (Rn0[3] - 3 * Rn0[1] * Rn1[2]);
                    break;
                case 4:
                    B[0] += 4 * k * (Rn0[3] * Rn1[1] - Rn0[1] * Rn1[3]);
                    B[1] += k * (Rn0[4] - 6 * Rn0[2] * Rn1[2] + Rn1[4]);
                    break;
                default: {
                    double pm = 1, Bx = 0.0, By = 0.0;
                    for (int j = 1; j <= (i + 1) / 2; ++j) {
                        Bx += pm * k * (Rn0[i - 2 * j + 1] * fact[i - 2 * j + 1] * Rn1[2 * j - 1] * fact[2 * j - 1]);
                        By += pm * k * (Rn0[i - 2 * j + 2] * fact[i - 2 * j + 2] * Rn1[2 * j - 2] * fact[2 * j - 2]);
                        pm *= -1;
                    }
                    if ((i + 1) / 2 == i / 2) {
                        const int j = (i + 2) / 2;
                        By += pm * k * (Rn0[i - 2 * j + 2] * fact[i - 2 * j + 2] * Rn1[2 * j - 2] * fact[2 * j - 2]);
                    }
                    B[0] += Bx;
                    B[1] += By;
                }
            }
        } else {
            switch (i) {
                case 0:
                    B[0] -= k;
                    break;
                case 1:
                    B[0] -= k * R[0];
                    B[1] += k * R[1];
                    break;
                case 2:
                    B[0] -= k * (Rn0[2] - Rn1[2]);
                    B[1] += 2 * k * R[0] * R[1];
                    break;
                case 3:
                    B[0] -= k * (Rn0[3] - 3 * Rn0[1] * Rn1[2]);
                    B[1] += k * (3 * Rn0[2] * Rn1[1] - Rn1[3]);
                    break;
                case 4:
                    B[0] -= k * (Rn0[4] - 6 * Rn0[2] * Rn1[2] + Rn1[4]);
                    B[1] += 4 * k * (Rn0[3] * Rn1[1] - Rn0[1] * Rn1[3]);
                    break;
                default: {
                    double pm = 1, Bx = 0, By = 0;
                    for (int j = 1; j <= (i + 1) / 2; ++j) {
                        Bx -= pm * k * (Rn0[i - 2 * j + 2] * fact[i - 2 * j + 2] * Rn1[2 * j - 2] * fact[2 * j - 2]);
                        By += pm * k * (Rn0[i - 2 * j + 1] * fact[i - 2 * j + 1] * Rn1[2 * j - 1] * fact[2 * j - 1]);
                        pm *= -1;
                    }
                    if ((i + 1) / 2 == i / 2) {
                        const int j = (i + 2) / 2;
                        Bx -= pm * k * (Rn0[i - 2 * j + 2] * fact[i - 2 * j + 2] * Rn1[2 * j - 2] * fact[2 * j - 2]);
                    }
                    B[0] += Bx;
                    B[1] += By;
                }
            }
        }
        Rn0[i + 1] = Rn0[i] * R[0];
        Rn1[i + 1] = Rn1[i] * R[1];
        fact[i + 1] = fact[i] / (i + 1);
    }
}

// Multipole::apply (Multipole.cpp:352-366) for R in the element frame: a
// field only for 0 <= z <= L and inside the elliptical aperture
// (ElementBase::isInsideTransverse, ElementBase.h:627-640; OPAL's default
// 0.5 m x 0.5 m, OpalElement.cpp:225-226); the reference particle's field
// (applyToReferenceParticle :377-397) with every component less its error.
SC_HD void multipole_field(const MapElem& e, const double* R, bool ref_particle, double* B) {
    if (R[2] < 0.0 || R[2] > e.range) return;
    const double ax = R[0] / e.aperture[0], ay = R[1] / e.aperture[1];
    if (!(ax * ax + ay * ay < 1.0)) return;
    const int nn = e.accuracy, ns = e.nskew;
    double c[kMaxMultipoleOrder];
    for (int i = 0; i < nn; ++i) c[i] = ref_particle ? e.coefs[i] - e.coefs[nn + i] : e.coefs[i];
    multipole_terms(c, nn, false, R, B);
    for (int i = 0; i < ns; ++i)
        c[i] = ref_particle ? e.coefs[2 * nn + i] - e.coefs[2 * nn + ns + i] : e.coefs[2 * nn + i];
    multipole_terms(c, ns, true, R, B);
}

// computeExternalFields (ParallelTTracker.cpp:614-643) for the elements of
// the table at time t: R in the reference frame -> lab (ref_to_lab) ->
// element frame (minus ELEMEDGE along z); each element's E and B rotated
// back and added to Ef, Bf.  ref_particle: the reference particle's fields
// (updateReferenceParticle, :1134-1155).
SC_HD void add_external_fields(const MapElem* el, int n, const Trafo& ref_to_lab, const double* R, double t, double* Ef,
                               double* Bf, bool ref_particle = false) {
    for (int k = 0; k < n; ++k) {
        double lab[3], loc[3], El[3] = {0.0, 0.0, 0.0}, Bl[3] = {0.0, 0.0, 0.0}, Er[3], Br[3];
        trafo_transform_to(ref_to_lab, R, lab);
        loc[0] = lab[0] - 0.0;
        loc[1] = lab[1] - 0.0;
        loc[2] = lab[2] - el[k].edge;
        if (el[k].kind == kElemRfCavity) {
            if (el[k].map3d)
                rfcavity3d_field(el[k], loc, t, El, Bl);
            else if (el[k].map2d)
                rfcavity2d_field(el[k], loc, t, El, Bl);
            else
                rfcavity_field(el[k], loc, t, El, Bl);
            trafo_rotate_from(ref_to_lab, El, Er);
            Ef[0] += Er[0];
            Ef[1] += Er[1];
            Ef[2] += Er[2];
        } else if (el[k].kind == kElemMultipole) {
            multipole_field(el[k], loc, ref_particle, Bl);
        } else if (el[k].map2d) {
            solenoid2d_field(el[k], loc, Bl);
        } else {
            solenoid_field(el[k], loc, Bl);
        }
        trafo_rotate_from(ref_to_lab, Bl, Br);
        Bf[0] += Br[0];
        Bf[1] += Br[1];
        Bf[2] += Br[2];
    }
}

// ---------------------------------------------------------------- pusher
// BorisPusher::push between switchToUnitlessPositions / switchOff...
SC_HD void push_one(double* R, const double* P, double dt) {
    const double s = kC * dt;
    double r0 = R[0] / s, r1 = R[1] / s, r2 = R[2] / s;
    double g = sqrt(1.0 + dot3(P, P));
    r0 += 0.5 * P[0] / g;
    r1 += 0.5 * P[1] / g;
    r2 += 0.5 * P[2] / g;
    R[0] = r0 * s;
    R[1] = r1 * s;
    R[2] = r2 * s;
}
// BorisPusher::kick
SC_HD void kick_one(double* P, const double* Ef, const double* Bf, double dt, double mass, double charge) {
    const double ke = 0.5 * dt * charge * kC / mass;
    P[0] += ke * Ef[0];
    P[1] += ke * Ef[1];
    P[2] += ke * Ef[2];
    const double gamma = sqrt(1.0 + dot3(P, P));
    const double kt = 0.5 * dt * charge * kC * kC / (gamma * mass);
    double t[3] = {kt * Bf[0], kt * Bf[1], kt * Bf[2]};
    double w[3], c[3];
    cross3(P, t, c);
    w[0] = P[0] + c[0];
    w[1] = P[1] + c[1];
    w[2] = P[2] + c[2];
    const double ks = 2.0 / (1.0 + dot3(t, t));
    double s[3] = {ks * t[0], ks * t[1], ks * t[2]};
    cross3(w, s, c);
    P[0] += c[0];
    P[1] += c[1];
    P[2] += c[2];
    P[0] += ke * Ef[0];
    P[1] += ke * Ef[1];
    P[2] += ke * Ef[2];
}

// ---------------------------------------------------------------- Green's function
// G at grid point (i, j, k) from the IGF antiderivative tmp on the (n0+2) x
// (n1+2) x (n2+2) grid: the 8-corner difference of FFTPoissonSolver.cpp
// :508-516 in its order, with G[0,0,0] <- G[0,0,1] (mirrorRhoField, :657).
// t0 = n0 + 2, t1 = n1 + 2.
SC_HD double igf_G_at(const double* __restrict__ tmp, int t0, int t1, int i, int j, int k) {
    if (i == 0 && j == 0 && k == 0) k = 1;
    auto T = [&](int a, int b, int e) { return tmp[(size_t)a + (size_t)t0 * ((size_t)b + (size_t)t1 * e)]; };
    double g = T(i + 1, j + 1, k + 1);
    g += T(i + 1, j, k);
    g += T(i, j + 1, k);
    g += T(i, j, k + 1);
    g -= T(i + 1, j + 1, k);
    g -= T(i + 1, j, k + 1);
    g -= T(i, j + 1, k + 1);
    g -= T(i, j, k);
    return g;
}

// ---------------------------------------------------------------- division
// a / b, correctly rounded, from rb = RN(1/b): one product, then the
// remainder a - q0 b (exact with an FMA) corrects q0 (Markstein, IBM J. Res.
// Dev. 34(1), 1990).  With rb correctly rounded the result equals the IEEE
// quotient; operands near the ends of the exponent range take the division.
// Callers pass divisors of at least 2^-70 (mesh spacings, c dt, gamma), so
// only the quotient is checked: a tiny, zero or huge q0 takes the division,
// and a fast quotient (|q0| >= 2^-899) has |a| >= 2^-969, where the FMA
// remainder is exact (a subnormal dividend never reaches the product path).
// The range test reads the biased exponent of q0 from its high word on the
// integer units: |q0| in [2^-899, 2^900) (exponent field 124 .. 1922; zero,
// subnormals, infinities and NaN fall outside).
SC_HD bool quot_in_range(double q) {
#ifdef __CUDA_ARCH__
    const unsigned hi = (unsigned)__double2hiint(q);
#else
    unsigned long long bits = 0;
    __builtin_memcpy(&bits, &q, sizeof bits);
    const unsigned hi = (unsigned)(bits >> 32);
#endif
    return ((hi >> 20) & 0x7ffu) - 124u < 1799u;
}
SC_HD double div_rcp(double a, double b, double rb) {
    const double q0 = a * rb;
    if (!quot_in_range(q0)) return a / b;
    const double r = fma(-q0, b, a);
    return fma(r, rb, q0);
}

// div_rcp without the branch: `fast` is cleared when q0 is outside the range
// in which the result is the IEEE quotient.  Callers check `fast` once after
// a group of quotients and redo the group with divisions if it was cleared.
SC_HD double div_rcp_nc(double a, double b, double rb, bool& fast) {
    const double q0 = a * rb;
    fast = fast && quot_in_range(q0);
    const double r = fma(-q0, b, a);
    return fma(r, rb, q0);
}

// ---------------------------------------------------------------- CIC
// Lower grid point and normalised offset of a particle (IntCIC.h:818-858 with
// getVertexBelow, UniformCartesian.hpp:1025-1039, and getCellPosition,
// :1084-1097).  Returns false when a stencil point would leave the n^3 field;
// with pz (a DC beam) the z stencil may also reach the guard planes -1 and n
// (lower points -1 .. n-1).
SC_HD bool cic_locate(const double* hr, const double* origin, const int* n, const double* x, int* lgp,
                      double* dpos, int pz = 0) {
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
        int i = (int)((x[d] - origin[d]) / hr[d]);
        int ngp = (x[d] >= origin[d]) ? i : i - 1;
        double gpos = (ngp + 0.5) * hr[d] + origin[d];
        double delta = hr[d];
        int l = ngp;
        if (gpos > x[d]) {
            l = ngp - 1;
            gpos = gpos - delta;
        }
        double dp = x[d] - gpos;
        dp /= delta;
        const int g = d == 2 ? pz : 0;
        if (l < -g) {
            ok = false;
            l = -g;
        }
        if (l > n[d] - 2 + g) {
            ok = false;
            l = n[d] - 2 + g;
        }
        lgp[d] = l;
        dpos[d] = dp;
    }
    return ok;
}

// cic_locate with the reciprocals rhr[d] = RN(1 / hr[d]): same results.
SC_HD bool cic_locate_r(const double* hr, const double* rhr, const double* origin, const int* n, const double* x,
                        int* lgp, double* dpos, int pz = 0) {
    bool ok = true, fast = true;
    for (int d = 0; d < 3; ++d) {
        int i = (int)div_rcp_nc(x[d] - origin[d], hr[d], rhr[d], fast);
        int ngp = (x[d] >= origin[d]) ? i : i - 1;
        double gpos = (ngp + 0.5) * hr[d] + origin[d];
        double delta = hr[d];
        int l = ngp;
        if (gpos > x[d]) {
            l = ngp - 1;
            gpos = gpos - delta;
        }
        double dp = x[d] - gpos;
        dp = div_rcp_nc(dp, delta, rhr[d], fast);
        const int g = d == 2 ? pz : 0;
        if (l < -g) {
            ok = false;
            l = -g;
        }
        if (l > n[d] - 2 + g) {
            ok = false;
            l = n[d] - 2 + g;
        }
        lgp[d] = l;
        dpos[d] = dp;
    }
    if (!fast) return cic_locate(hr, origin, n, x, lgp, dpos, pz);
    return ok;
}

// The periodic particle boundary of a DC beam along z (ParticlePeriodicBCond,
// ParticleBConds.h:37-45), applied once by boundp's update() over the
// particle layout's domain, which follows the mesh: [origin, origin + h n)
// (RegionLayout::Repartition and getMeshDomain, RegionLayout.hpp:773-789,
// :871-896; ParticleSpatialLayout.hpp:296-297).
SC_HD double wrap_z(double t, double lo, double hi) {
    if (t < lo) return hi - (lo - t);
    if (t >= hi) return lo + (t - hi);
    return t;
}

// push_one with s = c dt and rs = RN(1/s) precomputed: same results.
SC_HD void push_r(double* R, const double* P, double s, double rs) {
    bool fast = true;
    double r0 = div_rcp_nc(R[0], s, rs, fast), r1 = div_rcp_nc(R[1], s, rs, fast), r2 = div_rcp_nc(R[2], s, rs, fast);
    const double g = sqrt(1.0 + dot3(P, P));
    const double rg = 1.0 / g;
    r0 += div_rcp_nc(0.5 * P[0], g, rg, fast);
    r1 += div_rcp_nc(0.5 * P[1], g, rg, fast);
    r2 += div_rcp_nc(0.5 * P[2], g, rg, fast);
    if (!fast) {
        r0 = R[0] / s + 0.5 * P[0] / g;
        r1 = R[1] / s + 0.5 * P[1] / g;
        r2 = R[2] / s + 0.5 * P[2] / g;
    }
    R[0] = r0 * s;
    R[1] = r1 * s;
    R[2] = r2 * s;
}

// kick_one with ke = 0.5 dt q c / m and ktn = 0.5 dt q c c precomputed.
SC_HD void kick_r(double* P, const double* Ef, const double* Bf, double ke, double ktn, double mass) {
    P[0] += ke * Ef[0];
    P[1] += ke * Ef[1];
    P[2] += ke * Ef[2];
    const double gamma = sqrt(1.0 + dot3(P, P));
    const double kt = ktn / (gamma * mass);
    double t[3] = {kt * Bf[0], kt * Bf[1], kt * Bf[2]};
    double w[3], c[3];
    cross3(P, t, c);
    w[0] = P[0] + c[0];
    w[1] = P[1] + c[1];
    w[2] = P[2] + c[2];
    const double ks = 2.0 / (1.0 + dot3(t, t));
    double s[3] = {ks * t[0], ks * t[1], ks * t[2]};
    cross3(w, s, c);
    P[0] += c[0];
    P[1] += c[1];
    P[2] += c[2];
    P[0] += ke * Ef[0];
    P[1] += ke * Ef[1];
    P[2] += ke * Ef[2];
}

// ---------------------------------------------------------------- mesh
// boundp (PartBunchBase.hpp:802-884) from the beam-frame bounds, then the
// scalars of computeSelfFields (PartBunch.cpp:493-511, 541-547, 641).
// Returns false when h <= 0.
SC_HD_COLD bool derive_mesh(StepState& s, const BunchConst& bc) {
    double rmin[3] = {s.bmin[0], s.bmin[1], s.bmin[2]};
    double rmax[3] = {s.bmax[0], s.bmax[1], s.bmax[2]};
    // a DC beam's z spans one period from the lowest particle, not enlarged
    // (PartBunchBase.hpp:813-814, :840-843)
    const int dims = bc.pz ? 2 : 3;
    if (bc.pz) {
        rmax[2] = rmin[2] + bc.period;
        s.hr[2] = bc.period / (bc.n[2] - 1);
        s.mesh_rmin[2] = rmin[2];
        s.mesh_rmax[2] = rmax[2];
    }
    for (int i = 0; i < dims; ++i) {
        double length = rmax[i] - rmin[i];
        if (length < 0) length = -length;
        if (length < 1e-10) {
            rmax[i] += 1e-10;
            rmin[i] -= 1e-10;
        } else {
            rmax[i] += bc.dh * length;
            rmin[i] -= bc.dh * length;
        }
        s.hr[i] = (rmax[i] - rmin[i]) / (bc.n[i] - 1);
        s.mesh_rmin[i] = rmin[i];
        s.mesh_rmax[i] = rmax[i];
    }
    bool ok = s.hr[0] * s.hr[1] * s.hr[2] > 0;
    for (int i = 0; i < 3; ++i) s.origin[i] = rmin[i] - s.hr[i] / 2.0;
    for (int i = 0; i < 3; ++i) s.rhr[i] = 1.0 / s.hr[i];
    double gz = s.psum[2] / (double)bc.Ntot;
    gz *= gz;
    gz = sqrt(gz + 1.0);
    s.gammaz = gz;
    s.hr_scaled[0] = s.hr[0] * 1.0;
    s.hr_scaled[1] = s.hr[1] * 1.0;
    s.hr_scaled[2] = s.hr[2] * 1.0;
    s.hr_scaled[2] *= gz;
    s.tmp2 = 1 / s.hr_scaled[0] * 1 / s.hr_scaled[1] * 1 / s.hr_scaled[2];
    s.hvol = s.hr_scaled[0] * s.hr_scaled[1] * s.hr_scaled[2];
    s.betaC = sqrt(gz * gz - 1.0) / gz / kC;
    return ok;
}

// Beam-frame trafos of computeSpaceChargeFields (ParallelTTracker.cpp:550-554)
// from the momentum sum and the path length.  Returns false for an
// anti-parallel mean momentum.
SC_HD_COLD bool derive_beam_frame(StepState& s, const BunchConst& bc) {
    const double N = (double)bc.Ntot;
    double pmean[3] = {s.psum[0] / N, s.psum[1] / N, s.psum[2] / N};
    double zhat[3] = {0.0, 0.0, 1.0}, q[4];
    bool ok = get_quaternion(pmean, zhat, q);
    if (!ok) {
        q[0] = 1.0;
        q[1] = q[2] = q[3] = 0.0;
    }
    double qc[4] = {q[0], -q[1], -q[2], -q[3]};
    double org[3] = {0.0, 0.0, s.path_length};
    trafo_make(s.b2r, org, qc);
    s.r2b = s.b2r;
    trafo_invert(s.r2b);
    return ok;
}

// updateReferenceParticle + updateRefToLabCSTrafo (ParallelTTracker.cpp:1123-1212)
// with the elements of the table and an optional uniform B_z.
SC_HD bool advance_reference(StepState& s, const BunchConst& bc) {
    s.ref_to_lab_step = s.ref_to_lab;  // the particles' external fields use the frame of the step's start
    s.t_step = s.t;
    s.t += bc.dT;
    const double dt = s.t < bc.dT ? s.t : bc.dT;
    const double scaleFactor = kC * dt;
    double* rr = s.ref_R;
    double* rp = s.ref_P;
    double eref[3] = {0.0, 0.0, 0.0}, bref[3] = {0.0, 0.0, 0.0};
    for (int pass = 0; pass < 2; ++pass) {
        rr[0] /= scaleFactor;
        rr[1] /= scaleFactor;
        rr[2] /= scaleFactor;
        double g = sqrt(1.0 + dot3(rp, rp));
        rr[0] += 0.5 * rp[0] / g;
        rr[1] += 0.5 * rp[1] / g;
        rr[2] += 0.5 * rp[2] / g;
        rr[0] *= scaleFactor;
        rr[1] *= scaleFactor;
        rr[2] *= scaleFactor;
        if (pass == 0) {
            // updateReferenceParticle (ParallelTTracker.cpp:1134-1155): the
            // elements' fields at the reference particle at t - dt / 2, then
            // the kick
            add_external_fields(bc.sol, bc.nsol, s.ref_to_lab, rr, s.t - 0.5 * dt, eref, bref, true);
            if (bc.bz_ext != 0.0) bref[2] += bc.bz_ext;
            kick_one(rp, eref, bref, dt, bc.mass, bc.charge);
        }
    }
    s.path_length += sqrt(dot3(rr, rr));
    double zhat[3] = {0.0, 0.0, 1.0}, qu[4];
    bool ok = get_quaternion(rp, zhat, qu);
    if (!ok) {
        qu[0] = 1.0;
        qu[1] = qu[2] = qu[3] = 0.0;
    }
    trafo_make(s.upd, rr, qu);
    double v[3];
    trafo_transform_to(s.upd, rr, v);
    rr[0] = v[0];
    rr[1] = v[1];
    rr[2] = v[2];
    trafo_rotate_to(s.upd, rp, v);
    rp[0] = v[0];
    rp[1] = v[1];
    rp[2] = v[2];
    Trafo inv = s.upd;
    trafo_invert(inv);
    trafo_compose(s.ref_to_lab, inv);
    return ok;
}

}  // namespace sc
