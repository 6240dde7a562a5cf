/*
 * scgpu.h -- C ABI of the B200 space-charge step for OPAL's time-domain
 * tracker.  Plain C types only (pointers, sizes, doubles); no CUDA or torch
 * types cross this boundary.  Every entry point returns an int status
 * (SCGPU_OK or a negative SCGPU_ERR_*) and never aborts; the text of the
 * last failure is available from scgpu_last_error().
 *
 * Which reference interface each entry point replaces (paths relative to
 * the OPAL source tree):
 *
 *   scgpu_create / scgpu_destroy
 *       FieldSolver::initSolver -> new FFTPoissonSolver(mesh, layout,
 *       "INTEGRATED", bcz)  (src/Structure/FieldSolver.cpp:440-532, :486) and
 *       PartBunchBase::setSolver (src/Classic/Algorithms/PartBunchBase.hpp:1739-1754);
 *       device set-up of the DKS path ParallelTTracker::setupDKS /
 *       allocateDeviceMemory (src/Algorithms/ParallelTTracker.h:468-499)
 *   scgpu_compute_potential, scgpu_compute_potential_device
 *       virtual void PoissonSolver::computePotential(Field_t& rho, Vector_t hr)
 *       (src/Solvers/PoissonSolver.h:28; FFTPoissonSolver.cpp:337-382)
 *   scgpu_add_solenoid, scgpu_add_rfcavity, scgpu_clear_elements,
 *   scgpu_fieldmap_astra1d, scgpu_fieldmap_astra1d_dynamic, scgpu_fieldmap_2d,
 *   scgpu_fieldmap_3d
 *       ParallelTTracker::computeExternalFields (ParallelTTracker.cpp:595-643)
 *       with Solenoid::apply / Astra1DMagnetoStatic and RFCavity::apply /
 *       Astra1DDynamic (see below)
 *   scgpu_set_exchange
 *       the MPI reductions of a distributed bunch (get_bounds, calcMoments,
 *       the scatter into the distributed rho field) as an exchange callback
 *   scgpu_set_reorder_interval
 *       no counterpart (a tuning setting of this implementation's cell order)
 *   scgpu_kernels_per_step, scgpu_launch_count, scgpu_profile_track
 *       no counterpart (measurement of this implementation)
 *   scgpu_set_periodic_z
 *       the bcz argument of FFTPoissonSolver (FieldSolver BCFFTZ, src/Structure/FieldSolver.cpp:431, :486)
 *       with PartBunch::setBCForDCBeam (src/Classic/Algorithms/PartBunch.cpp:1079-1098)
 *   scgpu_add_multipole
 *       OpalMultipole::update (src/Elements/OpalMultipole.cpp:127-166) with Multipole::apply
 *       (src/Classic/AbsBeamline/Multipole.cpp:352-397) in computeExternalFields
 *   scgpu_set_beam_frequency
 *       PartBunchBase::setBeamFrequency (src/Classic/Algorithms/PartBunchBase.hpp:2535-2537)
 *   scgpu_compute_potential_image, scgpu_compute_potential_image_device
 *       virtual void PoissonSolver::computePotential(Field_t& rho, Vector_t hr, double zshift)
 *       (src/Solvers/PoissonSolver.h:59; FFTPoissonSolver.cpp:287-327 with
 *       shiftedIntGreensFunction :546-639 and mirrorRhoField(Field_t&) :667-693)
 *   scgpu_compute_self_fields
 *       PartBunch::computeSelfFields()  (src/Classic/Algorithms/PartBunch.cpp:482-647,
 *       declared PartBunchBase.h:372, called ParallelTTracker.cpp:583),
 *       preceded by boundp() (PartBunchBase.hpp:802-884)
 *   scgpu_compute_self_fields_binned
 *       the energy-bin loop of ParallelTTracker::computeSpaceChargeFields
 *       (ParallelTTracker.cpp:567-578): calcGammas (PartBunchBase.hpp:639-683),
 *       setBinCharge (:722-725) and PartBunch::computeSelfFields(int bin)
 *       (PartBunch.cpp:138-430) for every emitted bin, preceded by boundp()
 *   scgpu_set_energy_bins, scgpu_get_bin_gammas
 *       the Bin attribute and energy-bin state of PartBunchBase
 *       (weHaveEnergyBins :458-464, getLastEmittedEnergyBin :409-416,
 *       Rebin :432-446, getBinGamma :710-713) for the resident bunch of scgpu_track
 *   scgpu_bunch_upload / scgpu_bunch_download
 *       DKS writeDataAsync / readData of R, P  (ParallelTTracker.h:501-512, :514-529)
 *   scgpu_register_host / scgpu_unregister_host
 *       DKS registerHostMemory / unregisterHostMemory (ParallelTTracker.h:490-496)
 *   scgpu_track
 *       the ParallelTTracker::execute step loop (src/Algorithms/ParallelTTracker.cpp:343-388):
 *       timeIntegration1 (pushParticles / pushParticlesDKS, :434-447,
 *       ParallelTTracker.h:448-455, :514-529), computeSpaceChargeFields (:546-592),
 *       timeIntegration2 (kickParticles+pushParticles / kickParticlesDKS, :450-491,
 *       ParallelTTracker.h:442-446, :531-562), updateRefToLabCSTrafo (:1199-1212)
 *   scgpu_beam_parameters
 *       PartBunchBase::calcBeamParameters (PartBunchBase.hpp:1529-1614) with
 *       calcMoments (:2185-2259)
 *
 * Layouts: particle vectors are N x 3 doubles, x, y, z per particle (OPAL's
 * ParticleAttrib<Vector_t>).  Grids are nx*ny*nz doubles with x fastest:
 * index = i + nx*(j + ny*k), the cell-centred field of the reference without
 * its guard layer.
 *
 * Threading: one context per host thread; a context is not re-entrant.
 */
#ifndef SCGPU_H
#define SCGPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define SCGPU_ABI_VERSION 1

#define SCGPU_OK 0
#define SCGPU_ERR_ARG (-1)          /* invalid argument or size */
#define SCGPU_ERR_OOM (-2)          /* device or host allocation failed */
#define SCGPU_ERR_MESH (-3)         /* boundp: h <= 0, cannot build a mesh */
#define SCGPU_ERR_GUARD (-4)        /* a CIC stencil left the mesh */
#define SCGPU_ERR_FRAME (-5)        /* getQuaternion of an anti-parallel or null vector */
#define SCGPU_ERR_CUDA (-6)         /* CUDA runtime error */
#define SCGPU_ERR_STATE (-7)        /* call order (e.g. tracking without a bunch) */
#define SCGPU_ERR_UNSUPPORTED (-8)  /* mesh size or option this build does not support */
#define SCGPU_ERR_EXCHANGE (-9)     /* the exchange callback of a sharded bunch failed */

#define SCGPU_PLAIN_FP64 0  /* FP64 throughout */
#define SCGPU_MIXED 1       /* FP32 grid work, FP64 particles / Green's function / boost */

#define SCGPU_NSTATS 28     /* per-step statistics record: 27 moment sums + sum of gamma */

#define SCGPU_FIELD_RHO 0   /* charge density fed to the solver [C/m^3], nx*ny*nz */
#define SCGPU_FIELD_PHI 1   /* potential [V], nx*ny*nz */
#define SCGPU_FIELD_E 2     /* -grad(phi) scaled by (gz, gz, 1/gz) [V/m], 3*nx*ny*nz interleaved */

typedef struct scgpu_ctx scgpu_ctx;

/* FIELDSOLVER attributes (src/Structure/FieldSolver.cpp:127-165) */
typedef struct scgpu_solver_params {
    int mx, my, mt;          /* MX, MY, MT: mesh cells per axis (2n must factor into 2, 3, 5) */
    int precision;           /* SCGPU_PLAIN_FP64 or SCGPU_MIXED */
    double bboxincr;         /* BBOXINCR in percent (OPAL default 2.0) */
} scgpu_solver_params;

/* bunch constants and tracker state at upload */
typedef struct scgpu_bunch_params {
    double dT;               /* time step [s] */
    double mass;             /* rest energy [eV] (PartData::getM) */
    double charge;           /* particle charge [e] (PartData::getQ) */
    double q_macro;          /* charge per macro-particle [C] (PartBunch Q) */
    double coupling;         /* 1/(4 pi eps0) (TrackRun.cpp:423) */
    double bz_ext;           /* uniform external B_z [T] in the reference frame, 0 for a drift */
    double t;                /* time [s] */
    double path_length;      /* s-position of the reference particle [m] */
    double ref_R[3];         /* reference particle position (reference frame) */
    double ref_P[3];         /* reference particle beta*gamma */
} scgpu_bunch_params;

typedef struct scgpu_tracker_state {
    double t;
    double path_length;
    double ref_R[3];
    double ref_P[3];
    double q_macro;
    double ref_to_lab_origin[3];
    double ref_to_lab_quat[4];
    long long step;
} scgpu_tracker_state;

/* calcBeamParameters outputs */
typedef struct scgpu_beam_params {
    double rmean[3], pmean[3];
    double rrms[3], prms[3];
    double eps_norm[3], eps[3];
    double rprms[3];
    double gamma;
    double moments[27];      /* x, px, y, py, z, pz sums, then the lower triangle of products */
} scgpu_beam_params;

typedef struct scgpu_mesh {
    double hr[3];            /* mesh spacing of the last solve [m] */
    double origin[3];
    double rmin[3], rmax[3]; /* enlarged beam-frame bounds */
    double gammaz;
    double hr_scaled[3];     /* rest-frame spacing passed to the Poisson solve */
} scgpu_mesh;

int scgpu_abi_version(void);

int scgpu_create(scgpu_ctx** out, const scgpu_solver_params* params, int device);
void scgpu_destroy(scgpu_ctx* ctx);
const char* scgpu_last_error(const scgpu_ctx* ctx);
/* run on a caller-owned cudaStream_t (passed as void*); NULL = the context's own stream.
 * scgpu_track launches its step graphs on that stream; the kernels inside keep
 * the graph's own priorities (the main chain at the device's highest stream
 * priority, the Green's-function branch at the lowest), whatever the
 * priority of the caller's stream. */
int scgpu_set_stream(scgpu_ctx* ctx, void* cuda_stream);
int scgpu_synchronize(scgpu_ctx* ctx);

/* PoissonSolver::computePotential: rho (nx*ny*nz, x fastest) in, the open-
 * boundary convolution with the integrated Green's function out (in place),
 * i.e. phi * 4 pi eps0 / (hx hy hz) in the reference's units.  hr is the
 * rest-frame mesh spacing. */
int scgpu_compute_potential(scgpu_ctx* ctx, double* rho_inout, const double hr[3]);
/* the same on a device buffer of the context's GPU (device or managed memory
 * holding nx*ny*nz doubles); anything else returns SCGPU_ERR_ARG before any
 * work is enqueued */
int scgpu_compute_potential_device(scgpu_ctx* ctx, double* rho_inout_device, const double hr[3]);

/* PartBunch::computeSelfFields on a bunch already in the beam frame: boundp,
 * CIC deposit of q_macro*dT ... /dT, Poisson solve, -grad, CIC gather; writes
 * Ef, Bf (N x 3, beam frame).  *q_macro is updated by the reference's
 * Q *= dt ... Q /= dt round trip. */
int scgpu_compute_self_fields(scgpu_ctx* ctx, long long n, const double* R, const double* P, double* q_macro, double dT,
                              double* Ef, double* Bf);

/* Particle sharding over ranks (one context per GPU, each holding a shard of
 * one bunch; the reference distributes particles over MPI ranks and reduces
 * bounds, moments and the charge density across them: PartBunchBase.hpp:
 * 1178-1219 get_bounds, :2185-2259 calcMoments, IPPL's scatter into a
 * distributed field).  At fixed points of a step the library hands a
 * device buffer of this rank's partial results to `fn`, which combines it
 * over the ranks in place, on `cuda_stream` (e.g. ncclAllReduce), and
 * returns 0:
 *   SCGPU_EXCHANGE_MIN_F64  count doubles, elementwise minimum (bounds);
 *   SCGPU_EXCHANGE_SUM_U64  count 64-bit unsigned integers, sum modulo 2^64
 *                           (the deposit's fixed-point node sums and the
 *                           momentum / moment sums as 32-bit chunks).
 * Every combined value is exact, so the union of the shards evolves
 * bitwise as the whole bunch on one GPU.  total_particles is the bunch's
 * particle count over all ranks.  Call before scgpu_bunch_upload (the upload
 * combines the momentum sums); fn = NULL returns to a single-GPU bunch.
 * capturable = 1 when fn only enqueues stream work, so the step can be a
 * CUDA graph; otherwise steps are enqueued directly.  Energy bins, the
 * phase profile and scgpu_compute_self_fields are single-GPU only. */
#define SCGPU_EXCHANGE_SUM_U64 0
#define SCGPU_EXCHANGE_MIN_F64 1
typedef int (*scgpu_exchange_fn)(void* device_buffer, long long count, int op, void* cuda_stream, void* user);
int scgpu_set_exchange(scgpu_ctx* ctx, scgpu_exchange_fn fn, void* user, long long total_particles, int capturable);

/* Beamline elements with external fields, the step's computeExternalFields
 * (src/Algorithms/ParallelTTracker.cpp:595-643) and the reference
 * particle's (:1134-1155): SOLENOID elements (src/Classic/AbsBeamline/
 * Solenoid.cpp:163-215) with a 1D magnetostatic field map in ASTRA format
 * (src/Classic/Fields/Astra1DMagnetoStatic.cpp), at ELEMEDGE on a straight
 * beamline along z, scaled by KS [T].  Up to 8 elements; they add to the
 * uniform bz_ext of the bunch parameters.  scgpu_fieldmap_astra1d returns the
 * map's Fourier coefficients (2 accuracy - 1 of them), its first and last z
 * and the Fourier period, as Astra1DMagnetoStatic::readMap computes them. */
int scgpu_add_solenoid(scgpu_ctx* ctx, const char* fieldmap_path, double elemedge, double ks);
int scgpu_clear_elements(scgpu_ctx* ctx);
int scgpu_fieldmap_astra1d(const char* path, double* coefs, int max_coefs, int* ncoefs, double* zbegin, double* zend,
                           double* period);

/* RFCAVITY elements (src/Classic/AbsBeamline/RFCavity.cpp:232-310, built by
 * src/Elements/OpalCavity.cpp:150-195) with a 1D dynamic field map in ASTRA
 * format (src/Classic/Fields/Astra1DDynamic.cpp: header "AstraDynamic
 * <accuracy> [TRUE|FALSE]", the frequency in MHz, then "z Ez" lines), at
 * ELEMEDGE on a straight beamline along z, with VOLT [MV/m], FREQ [MHz] and
 * LAG [rad]: inside the map's z range the particles see
 * E += VOLT cos(omega t + LAG) E_map and B -= VOLT sin(omega t + LAG) B_map
 * at t = the step's start + dT / 2, the reference particle at the end of
 * the step - dT / 2 (ParallelTTracker.cpp:628, :1149).  They share the
 * table of 8 elements with the solenoids.  scgpu_fieldmap_astra1d_dynamic
 * returns the map's coefficients (scaled to V/m per MV/m), first and last z,
 * Fourier period and frequency [MHz]. */
int scgpu_add_rfcavity(scgpu_ctx* ctx, const char* fieldmap_path, double elemedge, double volt_mv_per_m,
                       double freq_mhz, double lag_rad);
int scgpu_fieldmap_astra1d_dynamic(const char* path, double* coefs, int max_coefs, int* ncoefs, double* zbegin,
                                   double* zend, double* period, double* frequency_mhz);

/* 2D field maps on an (r, z) grid in OPAL's own format: scgpu_add_solenoid
 * takes a 2DMagnetoStatic map (src/Classic/Fields/FM2DMagnetoStatic.cpp)
 * and scgpu_add_rfcavity a 2DDynamic map (FM2DDynamic.cpp) in place of the
 * ASTRA 1D ones, chosen by the file's first word as Fieldmap::getFieldmap
 * does.  Header "2DMagnetoStatic XZ|ZX [TRUE|FALSE]" or "2DDynamic XZ|ZX
 * [TRUE|FALSE]"; XZ: "zbegin zend nz" [cm, intervals], (dynamic) the
 * frequency [MHz], "rbegin rend nr", then (nz+1)(nr+1) lines r-major of
 * "Bz Br" or "Ez Er E Ht" [MV/m, A/m]; ZX: the r line first, z-major lines
 * "Br Bz" or "Er Ez Ht E".  The field is the reference's bilinear
 * interpolation at the particle's distance from the axis, B = KS (Br x/r,
 * Br y/r, Bz); E = VOLT cos(omega t + LAG) (Er x/r, Er y/r, Ez) and
 * B -= VOLT sin(omega t + LAG) (-Bt y/r, Bt x/r, 0); none outside the grid
 * (the reference also loses a particle beyond the map radially).
 * scgpu_fieldmap_2d reads a map as those elements do: *dynamic, the grid
 * points nz and nr, ranges = {zbegin, zend, rbegin, rend} [m], the
 * frequency [MHz] (dynamic), and, when values is not NULL, the normalised
 * values component-major (Bz, Br or Ez [V/m], Er [V/m], Bt [T]), value
 * (c, z i, r j) at values[(c nr + j) nz + i]; capacity counts doubles. */
int scgpu_fieldmap_2d(const char* path, int* dynamic, int* nz, int* nr, double* ranges, double* frequency_mhz,
                      double* values, long long capacity);

/* 3D field maps of RF cavities in OPAL's own format: scgpu_add_rfcavity
 * takes a 3DDynamic map (src/Classic/Fields/FM3DDynamic.cpp), chosen by the
 * file's first word.  Header "3DDynamic [TRUE|FALSE]", the frequency [MHz],
 * "xbegin xend nx", "ybegin yend ny", "zbegin zend nz" [cm, intervals], then
 * (nx+1)(ny+1)(nz+1) lines "Ex Ey Ez Hx Hy Hz" [MV/m, A/m], x outer, z
 * inner.  The field is the reference's trilinear interpolation
 * (FM3DDynamic::getFieldstrength) with E = VOLT cos(omega t + LAG) E_map and
 * B -= VOLT sin(omega t + LAG) B_map; none in the last two grid planes along
 * any axis (the reference loses a particle there transversely).  A 3D
 * magnetostatic map (FM3DMagnetoStatic) is refused: SCGPU_ERR_UNSUPPORTED.
 * scgpu_fieldmap_3d reads a map as the element does: the grid points n =
 * {nx, ny, nz}, ranges = {xbegin, xend, ybegin, yend, zbegin, zend} [m], the
 * frequency [MHz] and, when values is not NULL, the normalised values
 * component-major (Ex, Ey, Ez [V/m], Bx, By, Bz [T]), value (c, x i, y j,
 * z k) at values[c nx ny nz + (i ny + j) nz + k]; capacity counts doubles. */
int scgpu_fieldmap_3d(const char* path, int* n, double* ranges, double* frequency_mhz, double* values,
                      long long capacity);

/* MULTIPOLE (src/Elements/OpalMultipole.cpp:127-166 attributes L, KN, DKN,
 * KS, DKS and ELEMEDGE; src/Classic/AbsBeamline/Multipole.cpp): a straight
 * multipole at ELEMEDGE on the lab z axis with field for 0 <= z - ELEMEDGE
 * <= L.  kn[0..nkn) and ks[0..nks) are the normal and skew strengths of
 * orders 1 (dipole) .. 20 [T m^(1-n)], dkn / dks their errors (NULL: none);
 * each is stored as Multipole::setNormalComponent / setSkewComponent do
 * (:106-163, the dipole and sextupole halved, octupole and decapole
 * divided) and the field is Multipole::computeField (:229-349) in its
 * expression order.  The particles see components plus errors, the
 * reference particle components alone (applyToReferenceParticle,
 * :377-397).  OPAL's default aperture, an ellipse of 0.5 m semi-axes,
 * applies: outside it no field is added (the reference also marks such a
 * particle lost; particle removal is not part of this library).  At most 8
 * elements of all kinds. */
int scgpu_add_multipole(scgpu_ctx* ctx, double elemedge, double length, const double* kn, int nkn, const double* dkn,
                        const double* ks, int nks, const double* dks);

/* FIELDSOLVER BCFFTZ=PERIODIC (FFTPoissonSolver(..., bcz="PERIODIC"),
 * src/Solvers/FFTPoissonSolver.cpp:60, :130-155, :189-190, :661-662): the
 * context's Poisson solves (scgpu_compute_potential[_device],
 * scgpu_compute_self_fields, scgpu_track) double the grid in x and y only
 * and convolve cyclically along z with the integrated Green's function at
 * offsets [0, nz) (not mirrored in z).  Needs an even nz.
 *
 * The bunch becomes a DC beam, as TrackRun pairs a periodic-z solver with
 * PartBunch::setBCForDCBeam (src/Track/TrackRun.cpp:899-902,
 * src/Classic/Algorithms/PartBunch.cpp:1079-1098):
 *   - boundp's mesh (PartBunchBase.hpp:813-843): x and y as for an open
 *     bunch; z starts at the lowest particle, not enlarged, and spans the
 *     period length L: hz = L / (nz - 1), origin_z = zmin - hz / 2;
 *   - the periodic particle boundary along z (ParticlePeriodicBCond,
 *     ippl/src/Particle/ParticleBConds.h:37-45) over the mesh's domain
 *     [origin_z, origin_z + nz hz), applied once per step before the
 *     scatter; a wrapped position stays wrapped (the tracked bunch carries
 *     it, as the reference's does);
 *   - the scatter drops the charge that lands in the z guard planes -1 and
 *     nz (the reference's single-rank scatter does not carry guard cells
 *     into the field); the gather reads there the field's periodic images
 *     (PeriodicFace: plane nz is plane 0, plane -1 is plane nz-1).
 * Energy bins and image charges return SCGPU_ERR_UNSUPPORTED while it is on. */
int scgpu_set_periodic_z(scgpu_ctx* ctx, int periodic);

/* PartBunchBase::setBeamFrequency (src/Classic/Algorithms/PartBunchBase.hpp:
 * 2535-2537; TrackRun.cpp:496 passes the BEAM's FREQUENCY in Hz): the DC
 * beam's period length L = c / f.  Default L = c / 1 GHz (PartBunchBase.hpp:
 * 132).  f must be positive and finite. */
int scgpu_set_beam_frequency(scgpu_ctx* ctx, double f_hz);

/* How often the tracker puts the particle arrays in cell order (a counting
 * sort by the CIC cell, so that the deposit's warps share few cells): every
 * `steps` steps of scgpu_track, counted from the upload; 0 never (the
 * deposit then slows as the order decays; results do not change, the sums
 * are exact).  Default 32, or the environment variable SCGPU_REORDER_EVERY
 * at scgpu_create.  No counterpart in the reference, whose scatter runs in
 * storage order. */
int scgpu_set_reorder_interval(scgpu_ctx* ctx, int steps);

/* PoissonSolver::computePotential(rho, hr, zshift): rho in, the potential of
 * its image charge out (in place, same units as scgpu_compute_potential):
 * minus the convolution with the integrated Green's function shifted by
 * zshift along z, read back with z flipped (index k <- nz - 1 - k). */
int scgpu_compute_potential_image(scgpu_ctx* ctx, double* rho_inout, const double hr[3], double zshift);
int scgpu_compute_potential_image_device(scgpu_ctx* ctx, double* rho_inout_device, const double hr[3], double zshift);

/* Energy bins: bins[i] in [0, nbins) for particle i; the fields of bins
 * [0, min(last_emitted, nbins)) and of their image charges are summed; at
 * most 64 bins. */
#define SCGPU_MAX_BINS 64

/* The energy-bin loop of computeSpaceChargeFields on a bunch already in the
 * beam frame: boundp, calcGammas, then per emitted bin the CIC deposit of
 * its particles (charge q_macro each), the bin's own field and its image's
 * (the bin's gamma for the boost, its image shifted behind the cathode
 * plane z = 0); writes Ef, Bf (N x 3, beam frame, summed over the bins) and,
 * if bin_gamma is not NULL, the nbins bin gammas (1 for an empty bin).
 * q_macro is left unchanged (the reference restores Q after every bin). */
int scgpu_compute_self_fields_binned(scgpu_ctx* ctx, long long n, const double* R, const double* P, const int* bins,
                                     int nbins, int last_emitted, double q_macro, double dT, double* Ef, double* Bf,
                                     double* bin_gamma);

int scgpu_register_host(scgpu_ctx* ctx, void* ptr, long long bytes);
int scgpu_unregister_host(scgpu_ctx* ctx, void* ptr);

/* Bunch state (reference frame, coordinates relative to the reference
 * particle).  Upload resets the tracker state from *bp. */
int scgpu_bunch_upload(scgpu_ctx* ctx, long long n, const double* R, const double* P, const scgpu_bunch_params* bp);
int scgpu_bunch_download(scgpu_ctx* ctx, double* R, double* P);

/* Advance the device-resident bunch by nsteps ParallelTTracker steps.  When
 * stats is not NULL it receives nsteps records of SCGPU_NSTATS doubles: the
 * moment sums of the state at the end of each step (asynchronous copies;
 * pinned memory keeps them off the critical path). */
int scgpu_track(scgpu_ctx* ctx, int nsteps, double* stats);

/* Energy bins of the resident bunch: bins[i] is the bin of particle i in the
 * order of the last scgpu_bunch_upload (an upload clears them).  With
 * nbins > 0 scgpu_track computes the self fields by the energy-bin loop with
 * image charges; nbins == 0 returns to one solve (Distribution::Rebin).
 * The bins travel with the particles through the cell reorder. */
int scgpu_set_energy_bins(scgpu_ctx* ctx, const int* bins, int nbins, int last_emitted);
/* gammas (and, if count is not NULL, particle counts) of the nbins bins at the last step */
int scgpu_get_bin_gammas(scgpu_ctx* ctx, double* gamma, long long* count);

int scgpu_get_tracker_state(scgpu_ctx* ctx, scgpu_tracker_state* out);
int scgpu_beam_parameters(scgpu_ctx* ctx, scgpu_beam_params* out);
/* beam parameters from one SCGPU_NSTATS record of scgpu_track */
int scgpu_beam_parameters_from_stats(const double* record, long long n, scgpu_beam_params* out);

/* Statistics and particle files in the reference's formats.
 *
 * scgpu_stat_row: one row of the SDDS .stat file for the resident bunch
 * (DataSink::doWriteStatData, src/Structure/DataSink.cpp:281-449, after
 * calcBeamParameters, PartBunchBase.hpp:1529-1614): SCGPU_STAT_COLUMNS
 * values in the file's column order (t [ns], s, numParticles, charge, mean
 * energy [MeV], rms, emittances, means, reference particle, max extent,
 * correlations, dispersion, the external field at the reference particle,
 * energy spread, dt [ns], particles outside n sigma, particle 0).
 * scgpu_sdds_write_header / scgpu_sdds_append_row write the file
 * (header DataSink.cpp:585-1032; values as the reference's stream writes
 * them, %.15e followed by nine spaces and a tab); with_particle0 = 0 leaves
 * out the last six columns, as a multi-rank reference run does.
 * scgpu_read_fromfile[_count] / scgpu_write_fromfile: the ASCII distribution
 * of DISTRIBUTION TYPE=FROMFILE (Distribution.cpp:1074-1159): comment lines
 * ('#'), the count N, then N records "x px y py z pz"; momenta_in_ev
 * converts eV to beta*gamma (converteVToBetaGamma, :1047-1053). */
#define SCGPU_STAT_COLUMNS 48
int scgpu_stat_row(scgpu_ctx* ctx, double* row);
const char* scgpu_stat_column_name(int column);
int scgpu_sdds_write_header(const char* path, const char* input_name, int processors, const char* revision,
                            const char* flavor);
int scgpu_sdds_append_row(const char* path, const double* row, int with_particle0);
int scgpu_read_fromfile_count(const char* path, long long* n);
int scgpu_read_fromfile(const char* path, long long capacity, double* R, double* P, int momenta_in_ev, double mass_ev,
                        long long* n);
int scgpu_write_fromfile(const char* path, long long n, const double* R, const double* P);

/* diagnostics of the last solve: SCGPU_FIELD_* grids and the mesh */
int scgpu_get_field(scgpu_ctx* ctx, int which, double* out);
int scgpu_get_mesh(scgpu_ctx* ctx, scgpu_mesh* out);

/* device-side elapsed time of the last scgpu_track call [ms] */
double scgpu_last_track_ms(const scgpu_ctx* ctx);

/* Per-phase device timers, the counterpart of the reference's IpplTimings
 * ("SelfField total", "SF: GreensFTotal", "ComputePotential",
 * "TIntegration1/2", "Boundingbox"; ippl/src/Utility/IpplTimings.h:172-215,
 * PartBunchBase.hpp:2393-2397, FFTPoissonSolver.cpp:65-66).  Runs nsteps
 * tracking steps with the phases serialised on one stream and CUDA events
 * between them; phase_ms[SCGPU_NPHASES] receives the summed milliseconds. */
#define SCGPU_NPHASES 8
#define SCGPU_PHASE_DRIFT_BOUNDS 0   /* half drift, beam frame, bounds, mesh; reference particle */
#define SCGPU_PHASE_DEPOSIT 1        /* CIC charge deposit (exact node sums) */
#define SCGPU_PHASE_ASSEMBLE 2       /* node sums -> rho */
#define SCGPU_PHASE_GREEN 3          /* integrated Green's function + its spectrum */
#define SCGPU_PHASE_CONVOLUTION 4    /* pruned FFT convolution */
#define SCGPU_PHASE_GRAD 5
#define SCGPU_PHASE_GATHER_KICK 6    /* gather, frames, kick, drift, reference update */
#define SCGPU_PHASE_REORDER 7        /* cell-order sort of the particle arrays (every few steps) */
int scgpu_profile_track(scgpu_ctx* ctx, int nsteps, double* phase_ms);
/* number of kernels one tracking step launches (from the step's CUDA graph) */
int scgpu_kernels_per_step(scgpu_ctx* ctx);
/* kernels scgpu_track has launched on this context so far, reorder and
 * statistics steps included (the kernel nodes of the step graphs it ran);
 * SCGPU_ERR_UNSUPPORTED once a step ran outside a graph (a sharded bunch
 * with a host-side exchange).  No counterpart in the reference: the
 * benchmark's count of device launches. */
int scgpu_launch_count(scgpu_ctx* ctx, long long* kernels);

/* ------------------------------------------------------------------ batches
 * Many independent bunches that step together: every batched step launches
 * each kernel of the step once for all bunches (blocks index a device work
 * table of (bunch, block)), grouped by transform length for the FFT passes,
 * and the whole step is one CUDA graph launch while the membership is
 * unchanged.  This replaces running one tracker per design point, as the
 * reference's optimizer does (optimizer/Pilot/Worker.h:31-190 calling
 * OpalSimulation::run, src/Optimize/OpalSimulation.cpp:232); the reference
 * has no batched step.  Each bunch lives in its own context (a slot), so the
 * single-bunch calls (scgpu_bunch_download, scgpu_get_tracker_state,
 * scgpu_beam_parameters, scgpu_get_field) work on scgpu_batch_member().
 * Results do not depend on the batch's membership or tuning: all sums are
 * exact and no kernel mixes bunches.  A batch is not thread-safe. */
typedef struct scgpu_batch scgpu_batch;
/* precision: SCGPU_PLAIN_FP64 or SCGPU_MIXED for every bunch of the batch */
int scgpu_batch_create(scgpu_batch** out, int device, int precision);
void scgpu_batch_destroy(scgpu_batch* batch);
const char* scgpu_batch_last_error(const scgpu_batch* batch);
/* Adds a bunch (mesh from p; p->precision is ignored) and uploads it as
 * scgpu_bunch_upload does; returns its slot (>= 0) or a negative status. */
int scgpu_batch_add(scgpu_batch* batch, const scgpu_solver_params* p, long long n, const double* R, const double* P,
                    const scgpu_bunch_params* bp);
int scgpu_batch_remove(scgpu_batch* batch, int slot);
/* the context of an occupied slot (NULL otherwise); owned by the batch */
scgpu_ctx* scgpu_batch_member(scgpu_batch* batch, int slot);
int scgpu_batch_size(const scgpu_batch* batch);
/* every occupied slot advances nsteps ParallelTTracker steps */
int scgpu_batch_track(scgpu_batch* batch, int nsteps);
/* scgpu_batch_track in two halves: launch enqueues the steps and returns, so
 * the host can prepare and scgpu_batch_add further bunches (they join at the
 * next launch) while the device works; wait finishes the steps and reports
 * device errors.  Removing a slot waits for steps in flight. */
int scgpu_batch_launch(scgpu_batch* batch, int nsteps);
int scgpu_batch_wait(scgpu_batch* batch);
/* 1 when the launched steps have finished on the device (or none are in
 * flight), 0 while they run; never blocks.  A serving loop admits arriving
 * bunches while this is 0 and launches the next steps once it is 1, so the
 * device does not idle behind a long admission.  (No counterpart in the
 * reference: OPAL runs one simulation per process.) */
int scgpu_batch_done(scgpu_batch* batch);
/* Removed bunches leave their contexts (device buffers) parked for reuse by
 * later bunches on the same mesh; trim frees the parked ones. */
int scgpu_batch_trim(scgpu_batch* batch);
double scgpu_batch_last_track_ms(const scgpu_batch* batch);
/* Tuning of the batched launches: threads per block of the deposit (128,
 * 256 or 512) and, per transform length L, the FFT tile shape (0: the
 * widest, up to 256 threads per block; 1, 2, 3: a half, a quarter, an eighth
 * as many columns per block, down to one warp; 4: the y and x passes of 64-,
 * 128- and 256-point lines as register-resident line transforms, 8 threads
 * a line, the others as 0).  Untuned lengths take 4 where it applies, else
 * 0.  Every variant gives the same bits. */
int scgpu_batch_set_tuning(scgpu_batch* batch, int deposit_threads, int L, int fft_variant);
int scgpu_batch_get_tuning(const scgpu_batch* batch, int L, int* deposit_threads, int* fft_variant);
/* The autotuner: times trial_steps batched steps per candidate (deposit block
 * size, then the FFT tile shape of every transform length present) and keeps
 * the fastest.  The trial steps advance the bunches like scgpu_batch_track
 * (tuning never changes results); the number of steps taken is returned. */
int scgpu_batch_autotune(scgpu_batch* batch, int trial_steps);

/* The open-boundary Poisson solve of scgpu_compute_potential_device for
 * callers that cannot allocate device memory -- hosts whose device memory is
 * owned by their own pool allocator, or loops that cannot afford the device
 * synchronisation of cudaMalloc / cudaFree.  It has no counterpart in the
 * reference.  No context is needed and nothing is allocated: rho_dev
 * (nx*ny*nz doubles, x fastest) and phi_dev (same size; may equal rho_dev)
 * are the caller's device buffers on the current device (a host pointer, a
 * buffer of another GPU or one smaller than the mesh returns SCGPU_ERR_ARG
 * before anything is enqueued), and the scratch is a 4 MiB array inside the
 * library that every GPU loading the library keeps until the process exits.
 * Limits: at most 32 cells per axis (and 2n factoring into 2, 3, 5); larger
 * meshes return SCGPU_ERR_UNSUPPORTED.  The first call on a device sets it
 * up with the device current: it looks up the arrays' device addresses
 * (cudaGetSymbolAddress) and writes the library's twiddle table with one
 * synchronous copy; make that first call before any stream capture.  The
 * results are bitwise those of scgpu_compute_potential_device in the plain
 * form.  Every call shares the one scratch array, so calls that overlap on
 * the GPU (different streams, or several host threads) race; serialise them
 * on one stream.  The work is enqueued on cuda_stream (a cudaStream_t, NULL
 * for the default stream) and returns without synchronising.  A CUDA error
 * already pending in the calling thread is left in place and the call
 * returns SCGPU_ERR_CUDA without enqueuing anything; SCGPU_ERR_CUDA from a
 * failed launch of this call means its work may be partly enqueued. */
int scgpu_compute_potential_noalloc(const double* rho_dev, double* phi_dev, int nx, int ny, int nz,
                                    const double hr[3], void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif
