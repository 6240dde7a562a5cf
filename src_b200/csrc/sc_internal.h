// sc_internal.h -- launchers shared between the translation units of libscgpu.
#pragma once

#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "sc_common.cuh"

namespace sc {

// Device buffers of one bunch + solver instance.  All grid arrays use
// x-fastest order: index = x + n0 * (y + n1 * z).
struct DevBunch {
    BunchConst bc;
    int precision;  // 0 = plain FP64, 1 = mixed
    // particle state (SoA, beam or reference frame depending on the phase)
    double* x;
    double* y;
    double* z;
    double* px;
    double* py;
    double* pz;
    uint32_t* id;     // original index of the particle in each slot
    // sort
    uint32_t* keys;
    uint32_t* keys_alt;
    uint32_t* vals;
    uint32_t* vals_alt;
    int* hist;        // particles per cell (counting sort), zero between steps
    int* hist_scan;   // first sorted position of every cell
    int* scan_blocks; // chunk sums of the scan
    // deposit: fixed-point charge per node as (L, H), value H 2^32 + L; zero between steps
    unsigned long long* nacc;
    // 1: nacc holds sums of 26-bit fixed-point CIC weights (the mixed form's
    // deposit, in units of Q dt 2^-26); 0: fixed-point charges
    int dep_weights;
    // grids
    // T is double in the plain form and float in the mixed form.
    void* rho;        // n^3 real (T)
    double* phi;      // n^3 real, FP64 in both forms
    void* E4;         // n^3 x 4 (T): (-grad phi) * (g, g, 1/g), w unused
    void* spec;       // (n2+1) x L1 x L0 complex, FP64: the inverse half of the convolution
    void* spec_lo;    // same shape, complex float: forward half in the mixed form (null in the plain form)
    double* gtmp;     // (n0+2)(n1+2)(n2+2) IGF antiderivative
    double* gline;    // (n0+1)(n1+1)(n2+1) G then its cosine transforms (FP64)
    void* ghat;       // (n0+1)(n1+1)(n2+1) real spectrum of G (T)
    void* tw[3];      // twiddles exp(-2 pi i e / L_d), complex T, per axis
    // reductions
    double* partials;
    unsigned* ticket;
    StepState* st;
    int red_blocks;
    // per-launch scratch for optional outputs
    double* Ef;
    double* Bf;
    // energy bins (PartBunchBase.hpp:639-725); null / 0 for a bunch without
    int* bin;                        // energy bin of the particle in each slot
    int* bin_alt;                    // reorder scratch
    int nbins;                       // getNumberOfEnergyBins
    int nactive;                     // bins whose fields are computed: min(last emitted, nbins)
    StepState* bst;                  // per bin: this step's mesh scalars with the bin's gamma
    unsigned long long* nacc_bins;   // per active bin: node accumulators (as nacc)
    unsigned long long* bin_partials;
    double* F8;                      // n^3 x 8: summed E (x, y, z, -) and B (x, y, -, -) of every bin and image
    void* spec_fwd;                  // plain form with bins: forward spectrum kept for the image solve
    // image charge (FFTPoissonSolver.cpp:287-327, :546-639); null until used
    double* gtmp_img;                // 2 x (n0+2)(n1+2)(n2+2): antiderivative planes, z and z - n2 hz
    double* gimg;                    // 2 x (n0+1)(n1+1)(2 n2): the shifted G and its cosine transforms
    void* ghat_img;                  // (n2+1)(n1+1)(n0+1) complex T: minus the spectrum of the shifted G
                                     // (periodic z: the spectrum of the periodic G)
    int periodic_z;                  // BCFFTZ=PERIODIC: z not doubled, cyclic convolution along z
};

struct FftPlan {
    int L;
    int nst;
    int r[12];
};

FftPlan make_plan(int L);

// A buffer a caller hands to a *_device entry point: device memory of
// `device` (or managed memory) holding at least `bytes` from p.  Checked
// before anything is enqueued, so a host or foreign pointer becomes
// SCGPU_ERR_ARG instead of an illegal-address fault on the GPU.  *why says
// what is wrong.
bool device_buffer_ok(const void* p, size_t bytes, int device, std::string* why);
// a 2D (r, z) field map (sc_fieldmap.cpp): grid points, ranges [m], the
// frequency [MHz] of a dynamic map, and the values (Bz, Br or Ez, Er, Bt)
int fieldmap_2d(const char* path, bool* dynamic, int* nz, int* nr, double* zbegin, double* zend, double* rbegin,
                double* rend, double* freq_mhz, std::vector<double>* values);
// true when the map file's first word names a 2D map (2DMagnetoStatic / 2DDynamic)
bool fieldmap_is_2d(const char* path);
// 1 when the map file's first word names a 3D dynamic map (3DDynamic), 2 for
// a 3D magnetostatic one, else 0
int fieldmap_kind_3d(const char* path);
// a 3D dynamic map (sc_fieldmap.cpp): grid points {nx, ny, nz}, ranges
// {xbegin, xend, ybegin, yend, zbegin, zend} [m], the frequency [MHz] and the
// values (Ex, Ey, Ez [V/m], Bx, By, Bz [T], each (i ny + j) nz + k)
int fieldmap_3d(const char* path, int* n, double* ranges, double* freq_mhz, std::vector<double>* values);
int particle_grid(const DevBunch& b);
void prime_particle_grids();  // occupancy of the particle kernels, before any capture

// particle TU (sc_particles.cu)
void launch_reduce_state(const DevBunch& b, bool init_frame, cudaStream_t s);
// mixed: the mixed form's half drift and frame change (fused multiply-adds)
void launch_drift_to_beam(const DevBunch& b, bool drift, cudaStream_t s, bool mixed = false);
void launch_advance_reference(const DevBunch& b, cudaStream_t s);
void launch_cell_keys(const DevBunch& b, int digit_bits, cudaStream_t s);
void launch_deposit(const DevBunch& b, cudaStream_t s);
void launch_assemble_rho(const DevBunch& b, cudaStream_t s);
void launch_igf(const DevBunch& b, const double* hr_host, cudaStream_t s);
void launch_igf_tmp(const DevBunch& b, cudaStream_t s);  // the antiderivative alone
void launch_grad(const DevBunch& b, cudaStream_t s);
void launch_gather_kick_push(const DevBunch& b, bool stats, cudaStream_t s);
void launch_gather_fields(const DevBunch& b, cudaStream_t s);
void launch_reduce_stats(const DevBunch& b, cudaStream_t s);
void launch_aos_to_soa(const double* aos, double* a, double* b, double* c, long long n, cudaStream_t s);
// host order AoS -> slot order SoA: slot i takes particle id[i]
void launch_aos_to_soa_by_id(const double* aos, const uint32_t* id, double* a, double* b, double* c, long long n,
                             cudaStream_t s);
void launch_soa_to_aos(const double* a, const double* b, const double* c, double* aos, long long n, cudaStream_t s);
void launch_reorder(const DevBunch& b, cudaStream_t s);
void launch_iota(uint32_t* id, long long n, cudaStream_t s);
void launch_soa_to_aos_by_id(const double* a, const double* b, const double* c, const uint32_t* id, double* aos,
                             long long n, cudaStream_t s);
void launch_f64_to_f32(const double* in, float* out, long long n, cudaStream_t s);
void launch_f32_to_f64(const float* in, double* out, long long n, cudaStream_t s);
// sharded bunch: the reduction tails after the ranks' partials were combined
void launch_finish_mesh(const DevBunch& b, cudaStream_t s);
void launch_finish_psum(const DevBunch& b, bool frame, bool advance, cudaStream_t s);
void launch_finish_stats(const DevBunch& b, cudaStream_t s);
// statistics: bounds of the positions (out6 = min x, y, z, -max x, y, z) and one particle's state
void launch_bounds(const DevBunch& b, double* out6, cudaStream_t s);
void launch_find_id(const DevBunch& b, uint32_t target, double* out6, cudaStream_t s);

// energy bins (sc_particles.cu)
constexpr int kMaxBins = 64;
// calcGammas (PartBunchBase.hpp:639-683) into bst[b].gammaz, and the bin's
// solver scalars (PartBunch.cpp:173-185, :240-246) derived from this step's mesh
void launch_bin_gammas(const DevBunch& b, cudaStream_t s);
// one pass over the particles: the charge of every active bin into its own accumulators
void launch_deposit_bins(const DevBunch& b, cudaStream_t s);
// -grad phi of one bin's potential (view.phi) and of its image's (phi_img)
// (view.st = the bin's StepState), added into F8 in that order: E, and
// B = -+ betaC (E_y, -E_x) (PartBunch.cpp:238-244, image :417-427)
void launch_grad_acc(const DevBunch& view, const double* phi_img, cudaStream_t s);
void launch_gather_kick_push_bins(const DevBunch& b, bool stats, cudaStream_t s);
void launch_gather_fields_bins(const DevBunch& b, cudaStream_t s);
// bin of every slot from a host-order array (slot s holds particle id[s])
void launch_bins_by_id(const int* host_order, const uint32_t* id, int* bin, long long n, cudaStream_t s);
void launch_permute_bins(const DevBunch& b, cudaStream_t s);
// shifted antiderivative planes (st->hr_scaled, st->zshift) and the shifted G on (n0+1)(n1+1)(2 n2)
void launch_igf_image(const DevBunch& b, cudaStream_t s);

// Batched launches (many bunches, one kernel): `tab` is a device array of
// DevBunch; `items` holds one entry per bunch of the launch, (bunch, first
// block, blocks in x, blocks in y), sorted by first block; `nblocks` blocks
// are launched and each finds its bunch by a binary search over the items.
#ifdef __CUDACC__
__device__ __forceinline__ int4 resolve_block(const int4* __restrict__ items, int nitems) {
    const int blk = (int)blockIdx.x;
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&items[mid].y) <= blk)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int4 it = __ldg(&items[lo]);
    const int local = blk - it.y;
    // (bunch, block x, block y, blocks of the bunch)
    return make_int4(it.x, local % it.z, local / it.z, it.z * it.w);
}
#endif
enum : int {
    kBatchDrift = 0,
    kBatchPsum,
    kBatchStats,
    kBatchDeposit,
    kBatchAssemble,
    kBatchAdvance,
    kBatchIgfTmp,
    kBatchIgfG,
    kBatchGrad,
    kBatchGather,
};
void launch_batch(int kind, int precision, int threads, const DevBunch* tab, const int4* items, int nitems, int nblocks,
                  cudaStream_t s);

// FFT passes of a batch: every bunch of one launch has the same transform
// length L on the pass's axis; `variant` picks the tile shape (columns per
// block) the autotuner chose for that length.
enum : int {
    kPassZR2C = 0,   // A
    kPassYFwd,       // B
    kPassXConv,      // C
    kPassYInv,       // D
    kPassZC2R,       // E (self-field scaling)
    kPassDctZ,
    kPassDctY,
    kPassDctX,
    kNumPasses
};
constexpr int kFftVariants = 5;
constexpr int kFftLinesVariant = 4;  // register-resident line transforms for passes B, C, D (64/128/256 points)
bool fft_register_lines();           // line transforms enabled (SCGPU_FFT_LINES is not 0)
// Blocks of one pass for one bunch (grid x, y) with a tile-shape variant.
void fft_pass_grid(int pass, const DevBunch& b, int variant, int* gx, int* gy);
// Transform length of a pass's axis for a bunch.
int fft_pass_length(int pass, const DevBunch& b);
void launch_fft_pass_batch(int pass, int L, int precision, int variant, const DevBunch* tab, const int4* items,
                           int nitems, int nblocks, cudaStream_t s);

// sort TU (sc_sort.cu)
long long scan_scratch_ints(long long n);
void exclusive_scan(const int* in, int* out, long long n, int* blocks, cudaStream_t s);
void launch_sort(const DevBunch& b, cudaStream_t s);

// FFT TU (sc_fft.cu)
void launch_green_transform(const DevBunch& b, cudaStream_t s);
// Ĝ from the antiderivative alone (launch_igf_tmp): G is formed inside the
// first cosine transform; the same bits as launch_igf + launch_green_transform
void launch_green_transform_from_tmp(const DevBunch& b, cudaStream_t s);
void launch_convolution(const DevBunch& b, int mode, cudaStream_t s);
// the forward passes (A, B) need rho only; the rest (C, D, E) also the spectrum of G.
// The image part runs C, D, E with the shifted G's complex spectrum and
// writes phi with z flipped (FFTPoissonSolver.cpp:312-326).
enum : int { kConvForwardPart = 1, kConvRestPart = 2, kConvImagePart = 4 };
void launch_convolution_part(const DevBunch& b, int mode, int parts, cudaStream_t s);
// spectrum of the shifted G (b.gimg) into b.ghat_img
void launch_green_transform_image(const DevBunch& b, cudaStream_t s);
// periodic z: spectrum of G on its first n2 z planes (b.gline) into b.ghat_img
void launch_green_transform_periodic(const DevBunch& b, cudaStream_t s);
size_t fft_smem_bytes(const DevBunch& b);
void upload_twiddles(DevBunch& b, cudaStream_t s);
// the values upload_twiddles stores for transform length L (host)
void twiddle_values(int L, double2* td, float2* tf);
void fft_set_smem_limits();

// convolution modes
enum : int {
    kConvSelfField = 0,  // phi = conv * normFact * hvol * coupling (computeSelfFields)
    kConvPotential = 1,  // phi = conv * normFact (PoissonSolver::computePotential)
};

}  // namespace sc
