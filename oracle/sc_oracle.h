/*
 * sc_oracle.h -- CPU restatement of OPAL's space-charge step (test
 * infrastructure: the checker and the timed CPU baseline, never the product).
 */
#ifndef SC_ORACLE_H
#define SC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define SCO_ERR_ARG (-1)
#define SCO_ERR_OOM (-2)
#define SCO_ERR_MESH (-3)   /* boundp: h <= 0 (PartBunchBase.hpp:870-872) */
#define SCO_ERR_GUARD (-4)  /* a CIC stencil reached a guard cell */
#define SCO_ERR_FRAME (-5)  /* getQuaternion on an anti-parallel or null vector */

typedef struct {
    int nr[3];
    double hr[3];
    double origin[3];
    double rmin[3];
    double rmax[3];
} sco_mesh;

typedef struct {
    double origin[3];
    double quat[4];
    double M[9]; /* row-major rotation matrix */
} sco_trafo;

typedef struct {
    int nr[3];       /* MX, MY, MT: mesh cells per axis */
    int pad_;
    double dh;       /* BBOXINCR / 100 */
    double dT;       /* time step [s] */
    double mass;     /* rest energy [eV] */
    double charge;   /* particle charge [e] */
    double coupling; /* 1 / (4 pi eps0) */
    double bz_ext;   /* uniform external B_z [T] (0: drift) */
    double ref_pz;   /* reference particle beta*gamma along z at start */
    double period;   /* 0: open boundaries; > 0: DC beam (periodic z) with
                        this period length [m] (periodLength_m) */
} sco_params;

typedef struct {
    sco_params prm;
    double Q; /* macro-particle charge [C] */
    double t;
    double path_length;
    double ref_R[3];
    double ref_P[3];
    sco_trafo ref_to_lab;
    long long step;
} sco_tracker;

typedef struct {
    /* optional caller-owned outputs (NULL to skip) */
    double* rho; /* n^3: charge density fed to the solver [C/m^3] */
    double* phi; /* n^3: potential [V] */
    double* E;   /* 3 n^3 interleaved: -grad phi scaled by (g, g, 1/g) */
    double* Ef;  /* 3 N: E at particles, reference frame */
    double* Bf;  /* 3 N: B at particles, reference frame */
    /* filled by the call */
    sco_mesh mesh;
    double gammaz;
    double hr_scaled[3];
    double pmean[3];
    double rot_beam_to_ref[9];
    double update_origin[3];
} sco_debug;

typedef struct {
    double rmin[3], rmax[3];
    double rmean[3], pmean[3];
    double rrms[3], prms[3];
    double eps_norm[3], eps[3];
    double rprms[3];
    double gamma;
    double moments[27];
} sco_beam_params;

void sco_set_threads(int n);
int sco_get_threads(void);
int sco_max_threads(void);

double sco_const_c(void);
double sco_const_electron_mass_ev(void);
double sco_const_coupling(void);

int sco_get_quaternion(const double* u, const double* ref, double* q);
void sco_trafo_make(sco_trafo* t, const double* origin, const double* quat);
void sco_trafo_invert(sco_trafo* t);
void sco_trafo_compose(sco_trafo* t, const sco_trafo* right);
void sco_trafo_transform_to(const sco_trafo* t, const double* r, double* out);
void sco_trafo_rotate_to(const sco_trafo* t, const double* r, double* out);
void sco_quat_rotate(const double* q, const double* v, double* out);

void sco_push(long long n, double* R, const double* P, double dt);
void sco_kick(long long n, double* P, const double* Ef, const double* Bf, double dt, double mass, double charge);

void sco_bounds(long long n, const double* R, double* rmin, double* rmax);
void sco_moments(long long n, const double* R, const double* P, double* m27);
double sco_sum_gamma(long long n, const double* P);
void sco_beam_parameters_from_sums(const double* m27, double gsum, double N, sco_beam_params* bp);
int sco_beam_parameters(long long n, const double* R, const double* P, sco_beam_params* bp);

int sco_boundp(long long n, const double* R, const int* nr, double dh, sco_mesh* mesh);
int sco_scatter_cic(long long n, const double* R, double q, const sco_mesh* m, double* rho);
int sco_gather_cic(long long n, const double* R, const sco_mesh* m, const double* E, double* Ef);

/* DC beam (PartBunch::setBCForDCBeam, PartBunch.cpp:1079-1098; chosen for a
 * field solver with periodic z, TrackRun.cpp:899-902): boundp's mesh with z
 * not enlarged and spanning one period (PartBunchBase.hpp:813-843); the
 * periodic particle boundary along z (ParticlePeriodicBCond,
 * ParticleBConds.h:37-45) over the mesh's domain [origin, origin + n h);
 * CIC scatter dropping the charge that lands in the z guard layer and
 * gather reading the periodically filled guard layer. */
int sco_boundp_dc(long long n, const double* R, const int* nr, double dh, double period, sco_mesh* mesh);
void sco_wrap_z(long long n, double* R, const sco_mesh* mesh);
int sco_scatter_cic_dc(long long n, const double* R, double q, const sco_mesh* m, double* rho);
int sco_gather_cic_dc(long long n, const double* R, const sco_mesh* m, const double* E, double* Ef);

void sco_set_fft_engine(void* cffti, void* cfftf, void* cfftb, void* rffti, void* rfftf, void* rfftb);
int sco_fft_engine_is_own(void);
void sco_fft1d(int kind, long long n, double* data);
void sco_fft3d_r2c(const int* L, const double* in, double* out);
void sco_fft3d_c2r(const int* L, double* spec, double* out);

/* 0 (default): the reference's arithmetic -- host libm atan / log in the
 * Green's function, particle sums in storage order.  1: correctly rounded
 * atan / log (quad precision) and order-independent exact particle sums
 * (terms truncated at 2^-72, added as 128-bit integers, rounded once). */
void sco_set_exact(int on);
int sco_get_exact(void);
void sco_igf(const int* nr, const double* hr, double* G2);
int sco_compute_potential(const int* nr, double* rho, const double* hr);
void sco_neg_grad_scaled(const int* nr, const double* phi, const double* h, double gammaz, double* E);
/* R: beam-frame positions; a DC beam's (prm->period > 0) are wrapped along
 * z in place, as boundp's update() does */
int sco_compute_self_fields(const sco_params* prm, double* Q, long long n, double* R, const double* P,
                            double* Ef, double* Bf, sco_debug* dbg);

/* Elements with ASTRA 1D field maps: SOLENOID (kind 0; Solenoid.cpp:163-193,
 * Astra1DMagnetoStatic.cpp:162-196) and RFCAVITY (kind 1; RFCavity.cpp:
 * 232-270, Astra1DDynamic.cpp:192-229): the tracker adds their fields
 * (computeExternalFields, ParallelTTracker.cpp:614-643) */
#define SCO_MAX_ELEMENTS 8
#define SCO_MAX_MULTIPOLE 20
typedef struct {
    double edge, scale, zbegin, range, period;
    int accuracy;   /* map harmonics; MULTIPOLE (kind 2): normal components */
    int kind;
    double omega, phase, xlrep; /* RF: angular frequency, LAG, map's omega / c */
    int nskew;      /* MULTIPOLE: skew components */
    int map2d;      /* SOLENOID / RFCAVITY: 1 = a 2D (r, z) grid map */
    double aperture[2]; /* MULTIPOLE: elliptical aperture semi-axes [m] */
    int nz, nr;         /* 2D map: grid points along z and r */
    double hz, hr;      /* 2D map: spacings [m] */
    const double* grid; /* 2D map: Bz, Br or Ez, Er, Bt, each nz nr values, z fastest;
                           3D map: Ex, Ey, Ez, Bx, By, Bz, each nx ny nz values, (i ny + j) nz + k */
    int map3d, nx, ny, pad3_; /* RFCAVITY: 1 = a 3D (x, y, z) grid map; its points along x, y (nz above) */
    double hx, hy, xbegin, ybegin; /* 3D map: spacings and first grid x, y [m] */
    double coefs[255];  /* map coefficients; MULTIPOLE: normal, normal errors, skew, skew errors */
} sco_solenoid;
int sco_set_solenoids(const sco_solenoid* s, int n);
void sco_solenoid_field(const sco_solenoid* e, const double* R, double* B);
void sco_rfcavity_field(const sco_solenoid* e, const double* R, double t, double* E, double* B);
/* MULTIPOLE (kind 2; Multipole.cpp:106-163 component scaling, :229-349
 * computeField, :352-397 apply / applyToReferenceParticle): B at R (element
 * frame) added to B; ref_particle: components less their errors. */
void sco_multipole_field(const sco_solenoid* e, const double* R, int ref_particle, double* B);
/* SOLENOID with a 2D magnetostatic map (FM2DMagnetoStatic.cpp:158-189 with
 * Solenoid::apply) and RFCAVITY with a 2D dynamic map (FM2DDynamic.cpp:
 * 185-221 with RFCavity::apply): B (set) and E, B (added) at R, element frame */
void sco_solenoid2d_field(const sco_solenoid* e, const double* R, double* B);
void sco_rfcavity2d_field(const sco_solenoid* e, const double* R, double t, double* E, double* B);
/* RFCAVITY with a 3D dynamic map (FM3DDynamic.cpp:242-315 with
 * RFCavity::apply, RFCavity.cpp:232-250): E, B added at R, element frame */
void sco_rfcavity3d_field(const sco_solenoid* e, const double* R, double t, double* E, double* B);
/* Multipole::setNormalComponent / setSkewComponent (Multipole.cpp:106-163):
 * the stored component of order n (1 = dipole) from KN (or KS) and its error;
 * *err receives the stored error. */
double sco_multipole_component(int n, int skew, double v, double verr, double* err);

/* periodic z, BCFFTZ=PERIODIC (FFTPoissonSolver.cpp:60, :130-155, :661-662) */
void sco_igf_periodic_z(const int* nr, const double* hr, double* G2);
int sco_compute_potential_periodic_z(const int* nr, double* rho, const double* hr);

/* image charge (FFTPoissonSolver.cpp:287-327, :546-639) */
void sco_igf_shifted(const int* nr, const double* hr, double zshift, double* G2);
int sco_compute_potential_shifted(const int* nr, double* rho, const double* hr, double zshift);

/* energy bins (PartBunchBase.hpp:639-683; PartBunch.cpp:138-430;
 * ParallelTTracker.cpp:567-578) */
typedef struct {
    const int* bin;   /* per particle, in [0, nbins) */
    int nbins;        /* Distribution::getNumberOfEnergyBins */
    int last_emitted; /* Distribution::getLastEmittedEnergyBin */
} sco_bins;
int sco_bin_gammas(long long n, const double* P, const int* bin, int nbins, double* gamma, long long* count);
int sco_compute_self_fields_binned(const sco_params* prm, double qi, long long n, const double* R,
                                   const double* P, const int* bin, int nbins, int last_emitted,
                                   double* Ef, double* Bf, double* bin_gamma, sco_debug* dbg);

int sco_tracker_init(sco_tracker* tr, const sco_params* prm, double Q);
int sco_track(sco_tracker* tr, long long n, double* R, double* P, int nsteps, sco_debug* dbg);
int sco_track_binned(sco_tracker* tr, long long n, double* R, double* P, const int* bin, int nbins,
                     int last_emitted, int nsteps, sco_debug* dbg);

int sco_sizeof_tracker(void);
int sco_sizeof_debug(void);
int sco_sizeof_beam_params(void);

#ifdef __cplusplus
}
#endif
#endif
