// sc_api.cu -- the C ABI (include/scgpu.h): contexts, device memory, the step
// sequence and its CUDA graph.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "sc_ctx.h"

using namespace sc;

namespace sc {

// cuMemGetAddressRange from the driver, looked up once through the runtime
// (the library does not link the driver library itself).
using GetAddressRangeFn = int (*)(unsigned long long* base, size_t* size, unsigned long long ptr);
static GetAddressRangeFn address_range_fn() {
    static GetAddressRangeFn fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        cudaGetLastError();
        return reinterpret_cast<GetAddressRangeFn>(f);
    }();
    return fn;
}

bool device_buffer_ok(const void* p, size_t bytes, int device, std::string* why) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        *why = "not a pointer the CUDA runtime knows";
        return false;
    }
    if (a.type == cudaMemoryTypeDevice) {
        if (a.device != device) {
            *why = "device memory of another GPU";
            return false;
        }
    } else if (a.type != cudaMemoryTypeManaged) {
        *why = "host memory, not device memory";
        return false;
    }
    if (GetAddressRangeFn fn = address_range_fn()) {
        unsigned long long base = 0;
        size_t size = 0;
        const unsigned long long at = (unsigned long long)(uintptr_t)p;
        if (fn(&base, &size, at) == 0 && (at < base || at - base + bytes > size)) {
            *why = "allocation smaller than the mesh (" + std::to_string(size - (at - base)) + " bytes from the pointer, " +
                   std::to_string(bytes) + " needed)";
            return false;
        }
    }
    return true;
}

}  // namespace sc

namespace {

int fail(scgpu_ctx* c, int code, const std::string& what) {
    if (c) c->err = what;
    return code;
}

int cuda_fail(scgpu_ctx* c, cudaError_t e, const char* where) {
    return fail(c, SCGPU_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                          \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, #call); \
    } while (0)

template <typename P>
int dalloc(scgpu_ctx* c, P** p, size_t bytes) {
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(c, SCGPU_ERR_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return SCGPU_OK;
}

template <typename P>
void dfree(P*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

bool length_ok(int n) {
    if (n < 3 || 2 * n > 256) return false;
    return make_plan(2 * n).nst > 0;
}

// Particle arrays (the buffers that change size with the bunch) come from a
// per-device stream-ordered memory pool that keeps freed memory: resizing a
// context -- a serving loop reusing a parked context for a larger bunch --
// then costs no device-wide synchronisation, as cudaFree would, and steps in
// flight on other contexts keep running.
cudaMemPool_t particle_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[device]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t pool = nullptr;
        if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = pool;
    }
    return pools[device];
}

template <typename P>
int palloc(scgpu_ctx* c, P** p, size_t bytes) {
    cudaMemPool_t pool = particle_pool(c->device);
    if (!pool) return dalloc(c, p, bytes);
    if (bytes == 0) bytes = 16;
    cudaError_t e = cudaMallocFromPoolAsync((void**)p, bytes, pool, c->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        cudaGetLastError();
        return fail(c, SCGPU_ERR_OOM, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
    }
    return SCGPU_OK;
}

template <typename P>
void pfree(scgpu_ctx* c, P*& p) {
    if (p) {
        if (particle_pool(c->device))
            cudaFreeAsync((void*)p, c->stream);
        else
            cudaFree((void*)p);
    }
    p = nullptr;
}

void free_particles(scgpu_ctx* c) {
    DevBunch& b = c->b;
    pfree(c, b.x); pfree(c, b.y); pfree(c, b.z); pfree(c, b.px); pfree(c, b.py); pfree(c, b.pz); pfree(c, b.id);
    pfree(c, b.keys); pfree(c, b.keys_alt); pfree(c, b.vals); pfree(c, b.vals_alt);
    pfree(c, b.Ef); pfree(c, b.Bf);
    c->capacity = 0;
}

void drop_graphs(scgpu_ctx* c) {
    for (auto& row : c->graphs)
        for (auto& g : row) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
    for (auto& row : c->graphs_bins)
        for (auto& g : row) {
            if (g) cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

void free_bins(scgpu_ctx* c) {
    DevBunch& b = c->b;
    dfree(b.bin); dfree(b.bin_alt); dfree(b.bst); dfree(b.nacc_bins); dfree(b.bin_partials); dfree(b.F8);
    dfree(c->spec_fwd_buf); dfree(c->ghat_alt); dfree(c->ghat_img_alt); dfree(c->phi_img_buf);
    dfree(b.gtmp_img); dfree(b.gimg); dfree(b.ghat_img);
    for (int k = 0; k < kMaxBins; ++k) {
        if (c->ev_bin[k]) cudaEventDestroy(c->ev_bin[k]);
        if (c->ev_used[k]) cudaEventDestroy(c->ev_used[k]);
        c->ev_bin[k] = c->ev_used[k] = nullptr;
    }
    b.nbins = b.nactive = 0;
    c->bin_capacity = 0;
    c->bins_nbins_alloc = 0;
}

long long mesh_cells(const DevBunch& b) { return (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2]; }

// Buffers of the image-charge solve (FFTPoissonSolver.cpp:546-639).
int ensure_image(scgpu_ctx* c) {
    DevBunch& b = c->b;
    if (b.ghat_img) return SCGPU_OK;
    const long long n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long T3 = (n0 + 2) * (n1 + 2) * (n2 + 2);
    const long long GI = (n0 + 1) * (n1 + 1) * (2 * n2);
    const long long G3 = (n0 + 1) * (n1 + 1) * (n2 + 1);
    const size_t cs = b.precision == SCGPU_PLAIN_FP64 ? sizeof(double2) : sizeof(float2);
    int rc;
    if ((rc = dalloc(c, &b.gtmp_img, 2 * T3 * sizeof(double))) || (rc = dalloc(c, &b.gimg, 2 * GI * sizeof(double))) ||
        (rc = dalloc(c, (char**)&b.ghat_img, G3 * cs)))
        return rc;
    return SCGPU_OK;
}

// Buffers of the energy-bin loop for nbins bins and the current particle capacity.
int ensure_bins(scgpu_ctx* c, int nbins) {
    DevBunch& b = c->b;
    int rc = ensure_image(c);
    if (rc) return rc;
    const long long M = mesh_cells(b);
    const long long n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long S = (n2 + 1) * (2 * n1) * (2 * n0);
    const long long G3 = (n0 + 1) * (n1 + 1) * (n2 + 1);
    const size_t rs = b.precision == SCGPU_PLAIN_FP64 ? sizeof(double) : sizeof(float);
    const size_t cs = b.precision == SCGPU_PLAIN_FP64 ? sizeof(double2) : sizeof(float2);
    if (!b.bst) {
        if ((rc = dalloc(c, &b.bst, kMaxBins * sizeof(StepState))) ||
            (rc = dalloc(c, &b.bin_partials, 296 * kMaxBins * 8 * sizeof(unsigned long long))) ||
            (rc = dalloc(c, &b.F8, M * 8 * sizeof(double))) || (rc = dalloc(c, &c->phi_img_buf, M * sizeof(double))) ||
            (rc = dalloc(c, (char**)&c->ghat_alt, G3 * rs)) ||
            (rc = dalloc(c, (char**)&c->ghat_img_alt, G3 * cs)))
            return rc;
        if (b.precision == SCGPU_PLAIN_FP64 && (rc = dalloc(c, (char**)&c->spec_fwd_buf, S * sizeof(double2))))
            return rc;
        cudaMemsetAsync(b.bst, 0, kMaxBins * sizeof(StepState), c->stream);
        for (int k = 0; k < kMaxBins; ++k) {
            CK(cudaEventCreateWithFlags(&c->ev_bin[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&c->ev_used[k], cudaEventDisableTiming));
        }
    }
    if (c->bin_capacity < c->capacity) {
        dfree(b.bin);
        dfree(b.bin_alt);
        c->bin_capacity = 0;
        if ((rc = dalloc(c, &b.bin, c->capacity * sizeof(int))) || (rc = dalloc(c, &b.bin_alt, c->capacity * sizeof(int))))
            return rc;
        c->bin_capacity = c->capacity;
    }
    if (c->bins_nbins_alloc < nbins) {
        dfree(b.nacc_bins);
        c->bins_nbins_alloc = 0;
        if ((rc = dalloc(c, &b.nacc_bins, (size_t)nbins * M * 2 * sizeof(unsigned long long)))) return rc;
        CK(cudaMemsetAsync(b.nacc_bins, 0, (size_t)nbins * M * 2 * sizeof(unsigned long long), c->stream));
        c->bins_nbins_alloc = nbins;
    }
    return SCGPU_OK;
}

// The buffers one bin's solve works on: its StepState and accumulators, the
// kept forward spectrum, and one of two sets of Green's-function spectra.
DevBunch bin_view(const scgpu_ctx* c, int k) {
    DevBunch v = c->b;
    v.st = c->b.bst + k;
    v.nacc = c->b.nacc_bins + (size_t)2 * mesh_cells(c->b) * k;
    v.dep_weights = 0;  // the energy-bin deposit accumulates fixed-point charges
    v.spec_fwd = c->spec_fwd_buf;
    if (k & 1) {
        v.ghat = c->ghat_alt;
        v.ghat_img = c->ghat_img_alt;
    }
    return v;
}

// The energy-bin loop of computeSpaceChargeFields (ParallelTTracker.cpp:567-578)
// once the drift kernel has set this step's mesh: calcGammas, one deposit pass
// for all active bins, then per bin the charge density, the bin's own
// potential and its image's (computeSelfFields(bin), PartBunch.cpp:138-430),
// each field added into F8.  The Green's functions of a bin depend on its
// gamma only, so they run on the side stream, at most two bins ahead of the
// main stream's convolutions (two sets of spectra).
void enqueue_bins_fields(scgpu_ctx* c, cudaStream_t s) {
    DevBunch& b = c->b;
    const long long M = mesh_cells(b);
    launch_bin_gammas(b, s);
    cudaMemsetAsync(b.F8, 0, (size_t)M * 8 * sizeof(double), s);
    launch_deposit_bins(b, s);
    if (b.nactive <= 0) return;
    cudaEventRecord(c->ev_fork, s);
    cudaStreamWaitEvent(c->side, c->ev_fork, 0);
    for (int k = 0; k < b.nactive; ++k) {
        const DevBunch v = bin_view(c, k);
        if (k >= 2) cudaStreamWaitEvent(c->side, c->ev_used[k - 2], 0);
        launch_igf_tmp(v, c->side);
        launch_green_transform_from_tmp(v, c->side);
        launch_igf_image(v, c->side);
        launch_green_transform_image(v, c->side);
        cudaEventRecord(c->ev_bin[k], c->side);
        launch_assemble_rho(v, s);
        launch_convolution_part(v, kConvSelfField, kConvForwardPart, s);
        cudaStreamWaitEvent(s, c->ev_bin[k], 0);
        launch_convolution_part(v, kConvSelfField, kConvRestPart, s);
        DevBunch vi = v;  // the image's potential into its own buffer
        vi.phi = c->phi_img_buf;
        launch_convolution_part(vi, kConvSelfField, kConvImagePart, s);
        launch_grad_acc(v, c->phi_img_buf, s);
        cudaEventRecord(c->ev_used[k], s);
    }
}

int ensure_particles(scgpu_ctx* c, long long n) {
    if (n <= 0 || n > 0x7fffffffLL) return fail(c, SCGPU_ERR_ARG, "particle count must be in [1, 2^31)");
    DevBunch& b = c->b;
    if (n > c->capacity) {
        drop_graphs(c);
        free_particles(c);
        int rc;
        const size_t d = (size_t)n * sizeof(double);
        const size_t u = (size_t)n * sizeof(uint32_t);
        if ((rc = palloc(c, &b.x, d)) || (rc = palloc(c, &b.y, d)) || (rc = palloc(c, &b.z, d)) ||
            (rc = palloc(c, &b.px, d)) || (rc = palloc(c, &b.py, d)) || (rc = palloc(c, &b.pz, d)))
            return rc;
        if ((rc = palloc(c, &b.keys, u)) || (rc = palloc(c, &b.keys_alt, u)) || (rc = palloc(c, &b.vals, u)) ||
            (rc = palloc(c, &b.vals_alt, u)) || (rc = palloc(c, &b.id, u)))
            return rc;
        if ((rc = palloc(c, &b.Ef, 3 * d)) || (rc = palloc(c, &b.Bf, 3 * d))) return rc;
        c->capacity = n;
    }
    if (n != c->n) drop_graphs(c);
    c->n = n;
    b.bc.N = n;
    b.bc.sharded = c->xfn ? 1 : 0;
    b.bc.Ntot = c->xfn ? c->ntot : n;
    long long g = (n + 255) / 256;
    if (g < 1) g = 1;
    if (g > 148 * 8) g = 148 * 8;
    b.red_blocks = (int)g;
    return SCGPU_OK;
}

// One exchange of a sharded bunch; the first failure is kept for the caller.
void exchange(scgpu_ctx* c, void* buf, long long count, int op, cudaStream_t s) {
    const int rc = c->xfn(buf, count, op, (void*)s, c->xuser);
    if (rc != 0 && c->xerr == 0) c->xerr = rc;
}

int exchange_status(scgpu_ctx* c) {
    if (!c->xerr) return SCGPU_OK;
    const int rc = c->xerr;
    c->xerr = 0;
    return fail(c, SCGPU_ERR_EXCHANGE, "exchange callback returned " + std::to_string(rc));
}

// The momentum sums (and, with init_frame, the beam frame) of the whole
// bunch: reduce_state, then for a shard the exchange of the limbs.
void enqueue_psum(scgpu_ctx* c, bool init_frame, cudaStream_t s) {
    launch_reduce_state(c->b, init_frame, s);
    if (!c->xfn) return;
    exchange(c, c->b.st->xlimbs, 3 * 4, SCGPU_EXCHANGE_SUM_U64, s);
    launch_finish_psum(c->b, init_frame, false, s);
}

// The 27 moment sums and the sum of gamma of the whole bunch.
void enqueue_stats(scgpu_ctx* c, cudaStream_t s) {
    launch_reduce_stats(c->b, s);
    if (!c->xfn) return;
    exchange(c, c->b.st->xlimbs, 28 * 4, SCGPU_EXCHANGE_SUM_U64, s);
    launch_finish_stats(c->b, s);
}

// Puts the particle arrays in cell order: counting sort (keys, ranks, cell
// starts, scatter) and a gather of the particle arrays.
void enqueue_reorder(scgpu_ctx* c, cudaStream_t s) {
    DevBunch& b = c->b;
    launch_cell_keys(b, 0, s);
    launch_sort(b, s);
    launch_reorder(b, s);
    if (b.nbins > 0) launch_permute_bins(b, s);
    cudaMemsetAsync(b.hist, 0, (size_t)b.bc.n[0] * b.bc.n[1] * b.bc.n[2] * sizeof(int), s);
}

// The Green's function and its spectrum (open or periodic z), shared by the
// step and the solver entry points.
void enqueue_green(scgpu_ctx* c, cudaStream_t s) {
    if (c->b.periodic_z) {
        launch_igf(c->b, nullptr, s);
        launch_green_transform_periodic(c->b, s);
    } else {
        launch_igf_tmp(c->b, s);
        launch_green_transform_from_tmp(c->b, s);
    }
}

// one ParallelTTracker step on the context's stream
//   ref:  reference-particle update (needs only the tracker state; joins
//         before the gather, which applies its frame change)
//   main: drift -> deposit -> assemble [-> reorder] -> FFT A, B
//   side: (after the drift's mesh) Green's function, its spectrum
//   main: (join side) FFT C, D, E -> grad -> (join ref) gather/kick/push
// The branches write disjoint StepState fields.
void enqueue_step(scgpu_ctx* c, bool stats, bool reorder, cudaStream_t s) {
    DevBunch& b = c->b;
    const bool shard = c->xfn != nullptr;
    cudaEventRecord(c->ev_start, s);
    cudaStreamWaitEvent(c->ref, c->ev_start, 0);
    launch_advance_reference(b, c->ref);
    cudaEventRecord(c->ev_ref, c->ref);
    launch_drift_to_beam(b, true, s, b.precision != SCGPU_PLAIN_FP64);
    if (shard) {  // the bounds of all shards, then the mesh
        exchange(c, b.st->bnd6, 6, SCGPU_EXCHANGE_MIN_F64, s);
        launch_finish_mesh(b, s);
    }
    cudaEventRecord(c->ev_fork, s);
    cudaStreamWaitEvent(c->side, c->ev_fork, 0);
    enqueue_green(c, c->side);
    cudaEventRecord(c->ev_join, c->side);
    launch_deposit(b, s);
    if (shard)  // the charge of all shards: exact integer node sums
        exchange(c, b.nacc, 2 * mesh_cells(b), SCGPU_EXCHANGE_SUM_U64, s);
    launch_assemble_rho(b, s);
    if (reorder) enqueue_reorder(c, s);
    launch_convolution_part(b, kConvSelfField, kConvForwardPart, s);
    cudaStreamWaitEvent(s, c->ev_join, 0);
    launch_convolution_part(b, kConvSelfField, kConvRestPart, s);
    launch_grad(b, s);
    cudaStreamWaitEvent(s, c->ev_ref, 0);
    if (!shard) {
        launch_gather_kick_push(b, stats, s);
        return;
    }
    launch_gather_kick_push(b, false, s);
    exchange(c, b.st->xlimbs, 3 * 4, SCGPU_EXCHANGE_SUM_U64, s);
    launch_finish_psum(b, true, true, s);
    if (stats) enqueue_stats(c, s);
}

// The step with energy bins: the same branches, the self fields from the
// energy-bin loop, the gather reading the summed fields of all bins.
void enqueue_step_binned(scgpu_ctx* c, bool stats, bool reorder, cudaStream_t s) {
    DevBunch& b = c->b;
    cudaEventRecord(c->ev_start, s);
    cudaStreamWaitEvent(c->ref, c->ev_start, 0);
    launch_advance_reference(b, c->ref);
    cudaEventRecord(c->ev_ref, c->ref);
    launch_drift_to_beam(b, true, s);
    enqueue_bins_fields(c, s);
    if (reorder) enqueue_reorder(c, s);
    cudaStreamWaitEvent(s, c->ev_ref, 0);
    launch_gather_kick_push_bins(b, stats, s);
}

void enqueue_any_step(scgpu_ctx* c, bool stats, bool reorder, cudaStream_t s) {
    if (c->b.nbins > 0)
        enqueue_step_binned(c, stats, reorder, s);
    else
        enqueue_step(c, stats, reorder, s);
}

// Kernel nodes of a captured graph.
int graph_kernel_nodes(cudaGraph_t g) {
    size_t nn = 0;
    cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    cudaGraphGetNodes(g, nodes.data(), &nn);
    int kernels = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        cudaGraphNodeGetType(nd, &t);
        if (t == cudaGraphNodeTypeKernel) ++kernels;
    }
    return kernels;
}

int build_graph(scgpu_ctx* c, bool stats, bool reorder, cudaGraphExec_t* out) {
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
    enqueue_any_step(c, stats, reorder, c->own);
    cudaError_t e = cudaStreamEndCapture(c->own, &g);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaStreamEndCapture");
    (c->b.nbins > 0 ? c->graph_kernels_bins : c->graph_kernels)[stats ? 1 : 0][reorder ? 1 : 0] = graph_kernel_nodes(g);
    e = cudaGraphInstantiate(out, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
    return SCGPU_OK;
}

int status_from_flags(scgpu_ctx* c, int err) {
    if (!err) return SCGPU_OK;
    if (err & kFlagMesh) return fail(c, SCGPU_ERR_MESH, "boundp: h <= 0, cannot build a mesh");
    if (err & kFlagFrame) return fail(c, SCGPU_ERR_FRAME, "getQuaternion: anti-parallel or null vector");
    if (err & kFlagGuard) return fail(c, SCGPU_ERR_GUARD, "a CIC stencil left the mesh");
    if (err & kFlagSort) return fail(c, SCGPU_ERR_CUDA, "cell sort: scatter position out of range");
    if (err & kFlagBin) return fail(c, SCGPU_ERR_ARG, "an energy bin outside [0, nbins)");
    if (err & kFlagCopy) return fail(c, SCGPU_ERR_CUDA, "a bulk copy into shared memory did not complete");
    return fail(c, SCGPU_ERR_CUDA, "unknown device error flag");
}

int check_device_err(scgpu_ctx* c) {
    int err = 0;
    CK(cudaMemcpyAsync(&err, &c->b.st->err, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (err) {
        int zero = 0;
        cudaMemcpyAsync(&c->b.st->err, &zero, sizeof(int), cudaMemcpyHostToDevice, c->stream);
        cudaStreamSynchronize(c->stream);
    }
    return status_from_flags(c, err);
}

// calcBeamParameters from the moment sums (PartBunchBase.hpp:1529-1614)
int mom_idx(int i, int j) {
    if (i < j) {
        int t = i;
        i = j;
        j = t;
    }
    return 6 + i * (i + 1) / 2 + j;
}

void beam_params_from_sums(const double* m27, double gsum, double N, scgpu_beam_params* bp) {
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
        bp->rrms[i] = std::sqrt(rsqsum[i] / N);
        bp->prms[i] = std::sqrt(psqsum[i] / N);
        bp->eps_norm[i] = std::sqrt(eps2[i] > 0.0 ? eps2[i] : 0.0);
        double tmp = bp->rrms[i] * bp->prms[i];
        double fac = (tmp == 0) ? 0.0 : 1.0 / tmp;
        bp->rprms[i] = rpsum[i] * fac;
    }
    double gamma = gsum / N;
    bp->gamma = gamma;
    double den = gamma * std::sqrt(1.0 - 1.0 / (gamma * gamma));
    for (int i = 0; i < 3; ++i) bp->eps[i] = bp->eps_norm[i] / den;
    for (int k = 0; k < 27; ++k) bp->moments[k] = m27[k];
}

// With SCGPU_SYNC_CHECK set, every stage of the synchronous entry points is
// synchronised and checked, so a device error names the kernel that raised it.
bool sync_check_enabled() {
    static const bool on = std::getenv("SCGPU_SYNC_CHECK") != nullptr;
    return on;
}

int stage_check(scgpu_ctx* c, cudaStream_t s, const char* name) {
    if (!sync_check_enabled()) return SCGPU_OK;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(c, e, name);
    return SCGPU_OK;
}

#define STAGE(name)                                  \
    do {                                             \
        int rc_ = stage_check(c, s, name);           \
        if (rc_) return rc_;                         \
    } while (0)


}  // namespace

namespace sc {
int ctx_fail(scgpu_ctx* c, int code, const std::string& what) { return fail(c, code, what); }
void ctx_enqueue_reorder(scgpu_ctx* c, cudaStream_t s) { enqueue_reorder(c, s); }
int ctx_status_from_flags(scgpu_ctx* c, int flags) { return status_from_flags(c, flags); }
}  // namespace sc

extern "C" {

int scgpu_abi_version(void) { return SCGPU_ABI_VERSION; }

int scgpu_create(scgpu_ctx** out, const scgpu_solver_params* p, int device) {
    if (!out || !p) return SCGPU_ERR_ARG;
    *out = nullptr;
    if (p->precision != SCGPU_PLAIN_FP64 && p->precision != SCGPU_MIXED) return SCGPU_ERR_ARG;
    if (!length_ok(p->mx) || !length_ok(p->my) || !length_ok(p->mt)) return SCGPU_ERR_UNSUPPORTED;
    if (!(p->bboxincr >= 0.0)) return SCGPU_ERR_ARG;
    scgpu_ctx* c = new scgpu_ctx();
    c->device = device;
    c->sp = *p;
    c->use_graphs = std::getenv("SCGPU_NO_GRAPH") == nullptr;
    if (const char* r = std::getenv("SCGPU_REORDER_EVERY")) c->reorder_every = std::atoi(r);
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete c;
        return SCGPU_ERR_CUDA;
    }
    DevBunch& b = c->b;
    b.precision = p->precision;
    b.dep_weights = p->precision == SCGPU_MIXED ? 1 : 0;
    b.bc.n[0] = p->mx;
    b.bc.n[1] = p->my;
    b.bc.n[2] = p->mt;
    b.bc.dh = p->bboxincr / 100.0;
    b.bc.pz = 0;
    b.bc.period = kC / 1e9;  // periodLength_m's default (PartBunchBase.hpp:132)
    const long long n0 = p->mx, n1 = p->my, n2 = p->mt;
    const long long M = n0 * n1 * n2;
    int bits = 0;
    while ((1LL << bits) < M) ++bits;
    b.bc.key_bits = bits < 1 ? 1 : bits;
    const size_t rs = p->precision == SCGPU_PLAIN_FP64 ? sizeof(double) : sizeof(float);
    int rc = SCGPU_OK;
    const long long S = (n2 + 1) * (2 * n1) * (2 * n0);
    const long long T3 = (n0 + 2) * (n1 + 2) * (n2 + 2);
    const long long G3 = (n0 + 1) * (n1 + 1) * (n2 + 1);
    if ((rc = dalloc(c, &b.nacc, M * 2 * sizeof(unsigned long long))) ||
        (rc = dalloc(c, (char**)&b.rho, M * rs)) || (rc = dalloc(c, (char**)&b.phi, M * sizeof(double))) ||
        (rc = dalloc(c, (char**)&b.E4, 4 * M * rs)) || (rc = dalloc(c, (char**)&b.spec, S * sizeof(double2))) ||
        (p->precision != SCGPU_PLAIN_FP64 && (rc = dalloc(c, (char**)&b.spec_lo, S * sizeof(float2)))) ||
        (rc = dalloc(c, &b.gtmp, T3 * sizeof(double))) || (rc = dalloc(c, &b.gline, G3 * sizeof(double))) ||
        (rc = dalloc(c, (char**)&b.ghat, G3 * rs)) || (rc = dalloc(c, &b.st, sizeof(StepState))) ||
        (rc = dalloc(c, &b.partials, 148 * 8 * 32 * 16)) || (rc = dalloc(c, &b.ticket, 64)) ||
        (rc = dalloc(c, &b.hist, M * sizeof(int))) || (rc = dalloc(c, &b.hist_scan, M * sizeof(int))) ||
        (rc = dalloc(c, &b.scan_blocks, scan_scratch_ints(M) * sizeof(int)))) {
        scgpu_destroy(c);
        return rc;
    }
    for (int d = 0; d < 3; ++d) {
        const int L = 2 * b.bc.n[d];
        if ((rc = dalloc(c, (char**)&b.tw[d], L * (sizeof(double2) + sizeof(float2))))) {
            scgpu_destroy(c);
            return rc;
        }
    }
    // the step's main chain (captured on `own`) and the reference particle
    // at the highest priority, the Green's-function branch at the lowest, so
    // the branch fills the SMs the main chain leaves free (the step graphs
    // keep the priorities: cudaGraphInstantiateFlagUseNodePriority)
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    cudaStreamCreateWithPriority(&c->own, cudaStreamNonBlocking, prio_high);
    cudaStreamCreateWithPriority(&c->side, cudaStreamNonBlocking, prio_low);
    cudaStreamCreateWithPriority(&c->ref, cudaStreamNonBlocking, prio_high);
    c->stream = c->own;
    cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_start, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->ev_ref, cudaEventDisableTiming);
    cudaEventCreate(&c->ev_t0);
    cudaEventCreate(&c->ev_t1);
    cudaMemsetAsync(b.nacc, 0, M * 2 * sizeof(unsigned long long), c->own);
    cudaMemsetAsync(b.hist, 0, M * sizeof(int), c->own);
    cudaMemsetAsync(b.ticket, 0, 64, c->own);
    cudaMemsetAsync(b.st, 0, sizeof(StepState), c->own);
    fft_set_smem_limits();
    prime_particle_grids();
    upload_twiddles(b, c->own);
    e = cudaStreamSynchronize(c->own);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) {
        scgpu_destroy(c);
        return SCGPU_ERR_CUDA;
    }
    *out = c;
    return SCGPU_OK;
}

void scgpu_destroy(scgpu_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->own) cudaStreamSynchronize(c->own);
    if (c->stream && c->stream != c->own) cudaStreamSynchronize(c->stream);
    drop_graphs(c);
    free_particles(c);
    free_bins(c);
    dfree(c->d_elements);
    for (double*& g : c->map_grids) dfree(g);
    DevBunch& b = c->b;
    dfree(b.nacc); dfree(b.rho); dfree(b.phi); dfree(b.E4); dfree(b.spec); dfree(b.spec_lo);
    dfree(b.gtmp); dfree(b.gline); dfree(b.ghat); dfree(b.st); dfree(b.partials); dfree(b.ticket);
    dfree(b.hist); dfree(b.hist_scan); dfree(b.scan_blocks);
    for (int d = 0; d < 3; ++d) dfree(b.tw[d]);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->ev_t0) cudaEventDestroy(c->ev_t0);
    if (c->ev_t1) cudaEventDestroy(c->ev_t1);
    if (c->ev_start) cudaEventDestroy(c->ev_start);
    if (c->ev_ref) cudaEventDestroy(c->ev_ref);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->ref) cudaStreamDestroy(c->ref);
    if (c->own) cudaStreamDestroy(c->own);
    delete c;
}

const char* scgpu_last_error(const scgpu_ctx* c) { return c ? c->err.c_str() : "null context"; }

int scgpu_set_stream(scgpu_ctx* c, void* stream) {
    if (!c) return SCGPU_ERR_ARG;
    c->stream = stream ? (cudaStream_t)stream : c->own;
    return SCGPU_OK;
}

int scgpu_synchronize(scgpu_ctx* c) {
    if (!c) return SCGPU_ERR_ARG;
    CK(cudaStreamSynchronize(c->stream));
    return SCGPU_OK;
}

int scgpu_register_host(scgpu_ctx* c, void* ptr, long long bytes) {
    if (!c || !ptr || bytes <= 0) return SCGPU_ERR_ARG;
    CK(cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault));
    return SCGPU_OK;
}

int scgpu_unregister_host(scgpu_ctx* c, void* ptr) {
    if (!c || !ptr) return SCGPU_ERR_ARG;
    CK(cudaHostUnregister(ptr));
    return SCGPU_OK;
}

static int compute_potential_impl(scgpu_ctx* c, double* rho, const double hr[3], bool device_ptr) {
    if (!c || !rho || !hr) return fail(c, SCGPU_ERR_ARG, "null argument");
    for (int d = 0; d < 3; ++d)
        if (!(hr[d] > 0.0) || !std::isfinite(hr[d])) return fail(c, SCGPU_ERR_ARG, "hr must be positive and finite");
    CK(cudaSetDevice(c->device));
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    if (device_ptr) {
        std::string why;
        if (!device_buffer_ok(rho, (size_t)M * sizeof(double), c->device, &why))
            return fail(c, SCGPU_ERR_ARG, "rho_inout_device: " + why);
    }
    const cudaMemcpyKind in_kind = device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(b.st->hr_scaled, hr, 3 * sizeof(double), cudaMemcpyHostToDevice, s));
    if (b.precision == SCGPU_PLAIN_FP64) {
        CK(cudaMemcpyAsync(b.rho, rho, M * sizeof(double), in_kind, s));
    } else {
        double* stage = c->capacity * 3 >= M ? b.Ef : nullptr;
        bool tmp_alloc = false;
        if (!stage) {
            CK(cudaMalloc(&stage, M * sizeof(double)));
            tmp_alloc = true;
        }
        CK(cudaMemcpyAsync(stage, rho, M * sizeof(double), in_kind, s));
        launch_f64_to_f32(stage, (float*)b.rho, M, s);
        if (tmp_alloc) {
            CK(cudaStreamSynchronize(s));
            cudaFree(stage);
        }
    }
    enqueue_green(c, s);
    launch_convolution(b, kConvPotential, s);
    CK(cudaMemcpyAsync(rho, b.phi, M * sizeof(double), out_kind, s));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->have_solve = false;
    return SCGPU_OK;
}

// computePotential(rho, hr, zshift) (FFTPoissonSolver.cpp:287-327): the
// image charge's potential, through the shifted Green's function.
static int compute_potential_image_impl(scgpu_ctx* c, double* rho, const double hr[3], double zshift, bool device_ptr) {
    if (!c || !rho || !hr) return fail(c, SCGPU_ERR_ARG, "null argument");
    for (int d = 0; d < 3; ++d)
        if (!(hr[d] > 0.0) || !std::isfinite(hr[d])) return fail(c, SCGPU_ERR_ARG, "hr must be positive and finite");
    if (!std::isfinite(zshift)) return fail(c, SCGPU_ERR_ARG, "zshift must be finite");
    if (c->b.periodic_z) return fail(c, SCGPU_ERR_UNSUPPORTED, "image charges with periodic z");
    CK(cudaSetDevice(c->device));
    if (device_ptr) {
        std::string why;
        if (!device_buffer_ok(rho, (size_t)mesh_cells(c->b) * sizeof(double), c->device, &why))
            return fail(c, SCGPU_ERR_ARG, "rho_inout_device: " + why);
    }
    int rc = ensure_image(c);
    if (rc) return rc;
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    const long long M = mesh_cells(b);
    const cudaMemcpyKind in_kind = device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    CK(cudaMemcpyAsync(b.st->hr_scaled, hr, 3 * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(&b.st->zshift, &zshift, sizeof(double), cudaMemcpyHostToDevice, s));
    if (b.precision == SCGPU_PLAIN_FP64) {
        CK(cudaMemcpyAsync(b.rho, rho, M * sizeof(double), in_kind, s));
    } else {
        double* stage = nullptr;
        CK(cudaMalloc(&stage, M * sizeof(double)));
        cudaError_t e = cudaMemcpyAsync(stage, rho, M * sizeof(double), in_kind, s);
        if (e == cudaSuccess) launch_f64_to_f32(stage, (float*)b.rho, M, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaFree(stage);
        if (e != cudaSuccess) return cuda_fail(c, e, "staging rho");
    }
    launch_igf_image(b, s);
    launch_green_transform_image(b, s);
    launch_convolution_part(b, kConvPotential, kConvForwardPart | kConvImagePart, s);
    CK(cudaMemcpyAsync(rho, b.phi, M * sizeof(double), out_kind, s));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    c->have_solve = false;
    return SCGPU_OK;
}

// SOLENOID elements with ASTRA 1D magnetostatic maps on a straight beamline
// (Solenoid.cpp, Astra1DMagnetoStatic.cpp; ParallelTTracker::computeExternalFields).
static int upload_elements(scgpu_ctx* c) {
    DevBunch& b = c->b;
    drop_graphs(c);
    if (c->elements.empty()) {
        b.bc.sol = nullptr;
        b.bc.nsol = 0;
        return SCGPU_OK;
    }
    if (!c->d_elements) {
        int rc = dalloc(c, &c->d_elements, kMaxElements * sizeof(MapElem));
        if (rc) return rc;
    }
    CK(cudaMemcpyAsync(c->d_elements, c->elements.data(), c->elements.size() * sizeof(MapElem), cudaMemcpyHostToDevice,
                       c->stream));
    CK(cudaStreamSynchronize(c->stream));
    b.bc.sol = c->d_elements;
    b.bc.nsol = (int)c->elements.size();
    return SCGPU_OK;
}

// A 2D map's grid on the device, referenced by the element (freed with the
// context's elements).  want_dynamic: the element needs a dynamic (RF) map.
static int attach_map2d(scgpu_ctx* c, const char* path, bool want_dynamic, MapElem& e, double* freq_mhz) {
    bool dynamic = false;
    int nz = 0, nr = 0;
    double zb = 0, ze = 0, rb = 0, re = 0, f = 0;
    std::vector<double> v;
    int rc = fieldmap_2d(path, &dynamic, &nz, &nr, &zb, &ze, &rb, &re, &f, &v);
    if (rc) return fail(c, rc, std::string("cannot read the field map ") + path);
    if (dynamic != want_dynamic)
        return fail(c, SCGPU_ERR_ARG, std::string("the field map ") + path +
                                          (want_dynamic ? " is not a dynamic map" : " is not a magnetostatic map"));
    if (nz < 2 || nr < 2 || !(ze > zb) || !(re > rb)) return fail(c, SCGPU_ERR_ARG, "a 2D map needs two points per axis");
    CK(cudaSetDevice(c->device));
    double* d = nullptr;
    rc = dalloc(c, &d, v.size() * sizeof(double));
    if (rc) return rc;
    CK(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->map_grids.push_back(d);
    e.map2d = 1;
    e.nz = nz;
    e.nr = nr;
    e.hz = (ze - zb) / (nz - 1);  // FM2D*: (zend - zbegin) / intervals
    e.hr = (re - rb) / (nr - 1);
    e.grid = d;
    e.zbegin = zb;  // Solenoid / RFCavity::initialise: startField = zBegin, length = zEnd - zBegin
    e.range = ze - zb;
    if (freq_mhz) *freq_mhz = f;
    return SCGPU_OK;
}

// A 3D dynamic map's grid on the device (FM3DDynamic), referenced by the
// element as attach_map2d does.
static int attach_map3d(scgpu_ctx* c, const char* path, MapElem& e, double* freq_mhz) {
    int n[3] = {0, 0, 0};
    double r[6] = {0, 0, 0, 0, 0, 0}, f = 0.0;
    std::vector<double> v;
    int rc = fieldmap_3d(path, n, r, &f, &v);
    if (rc) return fail(c, rc, std::string("cannot read the field map ") + path);
    if (n[0] < 2 || n[1] < 2 || n[2] < 2 || !(r[1] > r[0]) || !(r[3] > r[2]) || !(r[5] > r[4]))
        return fail(c, SCGPU_ERR_ARG, "a 3D map needs two points per axis and increasing ranges");
    CK(cudaSetDevice(c->device));
    double* d = nullptr;
    rc = dalloc(c, &d, v.size() * sizeof(double));
    if (rc) return rc;
    CK(cudaMemcpy(d, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->map_grids.push_back(d);
    e.map3d = 1;
    e.nx = n[0];
    e.ny = n[1];
    e.nz = n[2];
    e.hx = (r[1] - r[0]) / (n[0] - 1);  // FM3DDynamic: (end - begin) / intervals
    e.hy = (r[3] - r[2]) / (n[1] - 1);
    e.hz = (r[5] - r[4]) / (n[2] - 1);
    e.xbegin = r[0];
    e.ybegin = r[2];
    e.grid = d;
    e.zbegin = r[4];  // RFCavity::initialise: startField = zbegin, length = zend - zbegin
    e.range = r[5] - r[4];
    *freq_mhz = f;
    return SCGPU_OK;
}

int scgpu_add_solenoid(scgpu_ctx* c, const char* fieldmap, double elemedge, double ks) {
    if (!c || !fieldmap) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!std::isfinite(elemedge) || !std::isfinite(ks)) return fail(c, SCGPU_ERR_ARG, "ELEMEDGE and KS must be finite");
    if ((int)c->elements.size() >= kMaxElements) return fail(c, SCGPU_ERR_UNSUPPORTED, "at most 8 elements");
    if (fieldmap_kind_3d(fieldmap) != 0)
        return fail(c, SCGPU_ERR_UNSUPPORTED, "3D magnetostatic maps are not supported (FM3DMagnetoStatic)");
    MapElem e{};
    if (fieldmap_is_2d(fieldmap)) {
        int rc = attach_map2d(c, fieldmap, false, e, nullptr);
        if (rc) return rc;
        e.edge = elemedge;
        e.scale = ks;
        e.kind = kElemSolenoid;
        CK(cudaStreamSynchronize(c->stream));
        c->elements.push_back(e);
        return upload_elements(c);
    }
    int ncoef = 0;
    int rc = scgpu_fieldmap_astra1d(fieldmap, e.coefs, kMaxSolCoefs, &ncoef, &e.zbegin, &e.range, &e.period);
    if (rc) return fail(c, rc, std::string("cannot read the field map ") + fieldmap);
    e.range = e.range - e.zbegin;  // zend - zbegin
    e.accuracy = (ncoef + 1) / 2;
    e.edge = elemedge;
    e.scale = ks;
    e.kind = kElemSolenoid;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    c->elements.push_back(e);
    return upload_elements(c);
}

// RFCAVITY with an ASTRA dynamic map (OpalCavity.cpp:150-195, RFCavity.cpp:
// 232-310).  The element's angular frequency is 1e6 * two_pi * FREQ
// (OpalCavity.cpp:159); when it differs from the map's by more than 1 % the
// map's is taken, as RFCavity::initialise does (:294-305).  The off-axis
// expansion uses the map's frequency (Astra1DDynamic.cpp:80-82).
int scgpu_add_rfcavity(scgpu_ctx* c, const char* fieldmap, double elemedge, double volt_mv_per_m, double freq_mhz,
                       double lag_rad) {
    if (!c || !fieldmap) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!std::isfinite(elemedge) || !std::isfinite(volt_mv_per_m) || !std::isfinite(lag_rad) || !(freq_mhz > 0.0) ||
        !std::isfinite(freq_mhz))
        return fail(c, SCGPU_ERR_ARG, "ELEMEDGE, VOLT and LAG must be finite and FREQ positive");
    if ((int)c->elements.size() >= kMaxElements) return fail(c, SCGPU_ERR_UNSUPPORTED, "at most 8 elements");
    MapElem e{};
    double fmap = 0.0;
    const int kind3d = fieldmap_kind_3d(fieldmap);
    if (kind3d == 2) return fail(c, SCGPU_ERR_ARG, std::string("the field map ") + fieldmap + " is not a dynamic map");
    if (kind3d == 1) {
        int rc = attach_map3d(c, fieldmap, e, &fmap);
        if (rc) return rc;
        if (!(fmap > 0.0)) return fail(c, SCGPU_ERR_ARG, "the 3D map's frequency must be positive");
    } else if (fieldmap_is_2d(fieldmap)) {
        int rc = attach_map2d(c, fieldmap, true, e, &fmap);
        if (rc) return rc;
        if (!(fmap > 0.0)) return fail(c, SCGPU_ERR_ARG, "the 2D map's frequency must be positive");
    } else {
        int ncoef = 0;
        int rc = scgpu_fieldmap_astra1d_dynamic(fieldmap, e.coefs, kMaxSolCoefs, &ncoef, &e.zbegin, &e.range, &e.period,
                                                &fmap);
        if (rc) return fail(c, rc, std::string("cannot read the field map ") + fieldmap);
        e.range = e.range - e.zbegin;  // zend - zbegin
        e.accuracy = (ncoef + 1) / 2;
    }
    e.edge = elemedge;
    e.scale = volt_mv_per_m;
    e.kind = kElemRfCavity;
    const double two_pi = 2 * kPi;
    const double omega_map = fmap * (two_pi * 1e6);
    double omega = 1e6 * two_pi * freq_mhz;
    if (std::fabs((omega - omega_map) / omega) > 0.01) omega = omega_map;
    e.omega = omega;
    e.phase = lag_rad;
    e.xlrep = omega_map / kC;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    c->elements.push_back(e);
    return upload_elements(c);
}

// Multipole::setNormalComponent / setSkewComponent (Multipole.cpp:106-163):
// the stored component of order n (1 = dipole) from KN or KS and its error,
// and the stored error.
static double multipole_component(int n, bool skew, double v, double verr, double* err) {
    double c, e;
    switch (n - 1) {
        case 0:  // dipole
            c = (v + verr) / 2;
            e = c;
            break;
        case 2:  // sextupole
            c = (v + verr) / 2;
            e = verr / 2;
            break;
        case 3:  // octupole
            c = skew ? (v + verr) / 6 : (v + verr) / 24;
            e = skew ? verr / 6 : verr / 24;
            break;
        case 4:  // decapole
            c = (v + verr) / 24;
            e = verr / 24;
            break;
        default:
            c = v + verr;
            e = verr;
    }
    *err = e;
    return c;
}

// MULTIPOLE (OpalMultipole::update, OpalMultipole.cpp:127-166: L, KN, DKN,
// KS, DKS; the errors padded with zeros to the components' count).
int scgpu_add_multipole(scgpu_ctx* c, double elemedge, double length, const double* kn, int nkn, const double* dkn,
                        const double* ks, int nks, const double* dks) {
    if (!c) return SCGPU_ERR_ARG;
    if (nkn < 0 || nks < 0 || nkn > kMaxMultipoleOrder || nks > kMaxMultipoleOrder || (nkn > 0 && !kn) ||
        (nks > 0 && !ks))
        return fail(c, SCGPU_ERR_ARG, "KN and KS hold 0 .. 20 components");
    if (!std::isfinite(elemedge) || !(length >= 0.0) || !std::isfinite(length))
        return fail(c, SCGPU_ERR_ARG, "ELEMEDGE must be finite and L finite and not negative");
    for (int i = 0; i < nkn; ++i)
        if (!std::isfinite(kn[i]) || (dkn && !std::isfinite(dkn[i]))) return fail(c, SCGPU_ERR_ARG, "KN, DKN must be finite");
    for (int i = 0; i < nks; ++i)
        if (!std::isfinite(ks[i]) || (dks && !std::isfinite(dks[i]))) return fail(c, SCGPU_ERR_ARG, "KS, DKS must be finite");
    if ((int)c->elements.size() >= kMaxElements) return fail(c, SCGPU_ERR_UNSUPPORTED, "at most 8 elements");
    MapElem e{};
    e.kind = kElemMultipole;
    e.edge = elemedge;
    e.range = length;
    e.accuracy = nkn;
    e.nskew = nks;
    e.aperture[0] = 0.5;  // OpalElement::getApert's default: ELLIPTICAL(0.5, 0.5)
    e.aperture[1] = 0.5;
    for (int i = 0; i < nkn; ++i)
        e.coefs[i] = multipole_component(i + 1, false, kn[i], dkn ? dkn[i] : 0.0, &e.coefs[nkn + i]);
    for (int i = 0; i < nks; ++i)
        e.coefs[2 * nkn + i] = multipole_component(i + 1, true, ks[i], dks ? dks[i] : 0.0, &e.coefs[2 * nkn + nks + i]);
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    c->elements.push_back(e);
    return upload_elements(c);
}

int scgpu_clear_elements(scgpu_ctx* c) {
    if (!c) return SCGPU_ERR_ARG;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    c->elements.clear();
    for (double*& g : c->map_grids) dfree(g);
    c->map_grids.clear();
    return upload_elements(c);
}

int scgpu_set_exchange(scgpu_ctx* c, scgpu_exchange_fn fn, void* user, long long total_particles, int capturable) {
    if (!c) return SCGPU_ERR_ARG;
    if (fn && total_particles <= 0) return fail(c, SCGPU_ERR_ARG, "total_particles must be positive");
    if (fn && c->b.nbins > 0) return fail(c, SCGPU_ERR_UNSUPPORTED, "energy bins of a sharded bunch");
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);
    c->xfn = fn;
    c->xuser = fn ? user : nullptr;
    c->ntot = fn ? total_particles : 0;
    c->xcapturable = fn && capturable;
    c->xerr = 0;
    c->b.bc.sharded = fn ? 1 : 0;
    c->b.bc.Ntot = fn ? total_particles : c->n;
    c->have_bunch = false;  // the bunch is uploaded again as a shard (or whole)
    return SCGPU_OK;
}

// setBeamFrequency (PartBunchBase.hpp:2535-2537, from the BEAM's FREQUENCY,
// TrackRun.cpp:496): the period length c / f of a DC beam.
int scgpu_set_beam_frequency(scgpu_ctx* c, double f_hz) {
    if (!c) return SCGPU_ERR_ARG;
    if (!(f_hz > 0.0) || !std::isfinite(f_hz)) return fail(c, SCGPU_ERR_ARG, "the beam frequency must be positive and finite");
    const double period = kC / f_hz;
    if (!std::isfinite(period) || !(period > 0.0)) return fail(c, SCGPU_ERR_ARG, "period length out of range");
    if (period == c->b.bc.period) return SCGPU_OK;
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    drop_graphs(c);  // the step graphs hold the bunch constants
    c->b.bc.period = period;
    return SCGPU_OK;
}

// Interval of the cell reorder in scgpu_track (0: never); the step graphs
// are keyed by whether a step reorders, so no graph is rebuilt.
int scgpu_set_reorder_interval(scgpu_ctx* c, int steps) {
    if (!c || steps < 0) return fail(c, SCGPU_ERR_ARG, "the reorder interval must be >= 0");
    c->reorder_every = steps;
    return SCGPU_OK;
}

// BCFFTZ=PERIODIC (FieldSolver.cpp:431, :486; FFTPoissonSolver.cpp:60,
// :130-155, :189-190, :661-662): the solves of this context use a grid
// doubled in x and y only and a cyclic convolution along z.  The resident
// bunch becomes a DC beam, as TrackRun selects setBCForDCBeam for a solver
// with periodic z (TrackRun.cpp:899-902; PartBunch.cpp:1079-1098): boundp's
// mesh spans one period along z and the particles wrap at the mesh's ends.
int scgpu_set_periodic_z(scgpu_ctx* c, int periodic) {
    if (!c) return SCGPU_ERR_ARG;
    DevBunch& b = c->b;
    const int on = periodic ? 1 : 0;
    if (on == b.periodic_z) return SCGPU_OK;
    if (on) {
        const int n2 = b.bc.n[2];
        if (n2 % 2 != 0 || n2 < 4 || make_plan(n2).nst <= 0)
            return fail(c, SCGPU_ERR_UNSUPPORTED, "periodic z needs an even mesh size along z with a supported transform");
        if (b.nbins > 0) return fail(c, SCGPU_ERR_UNSUPPORTED, "periodic z with energy bins");
    }
    CK(cudaSetDevice(c->device));
    CK(cudaStreamSynchronize(c->stream));
    if (on) {
        int rc = ensure_image(c);
        if (rc) return rc;
    }
    drop_graphs(c);
    b.periodic_z = on;
    b.bc.pz = on;
    upload_twiddles(b, c->stream);
    CK(cudaGetLastError());
    c->have_solve = false;
    return SCGPU_OK;
}

int scgpu_compute_potential_image(scgpu_ctx* c, double* rho, const double hr[3], double zshift) {
    return compute_potential_image_impl(c, rho, hr, zshift, false);
}

int scgpu_compute_potential_image_device(scgpu_ctx* c, double* rho, const double hr[3], double zshift) {
    return compute_potential_image_impl(c, rho, hr, zshift, true);
}

int scgpu_compute_potential(scgpu_ctx* c, double* rho, const double hr[3]) { return compute_potential_impl(c, rho, hr, false); }

int scgpu_compute_potential_device(scgpu_ctx* c, double* rho, const double hr[3]) {
    return compute_potential_impl(c, rho, hr, true);
}

int scgpu_compute_self_fields(scgpu_ctx* c, long long n, const double* R, const double* P, double* q_macro, double dT,
                              double* Ef, double* Bf) {
    if (!c || !R || !P || !q_macro || !Ef || !Bf) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (c->xfn) return fail(c, SCGPU_ERR_UNSUPPORTED, "self fields of a sharded bunch (use scgpu_track)");
    if (!(dT > 0.0)) return fail(c, SCGPU_ERR_ARG, "dT must be positive");
    CK(cudaSetDevice(c->device));
    int rc = ensure_particles(c, n);
    if (rc) return rc;
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    b.bc.dT = dT;
    if (b.bc.coupling == 0.0) b.bc.coupling = 1.0 / (4 * kPi * 8.854187817e-12);
    if (b.bc.mass == 0.0) b.bc.mass = 0.51099892e-03 * 1.0e9;
    bunch_constants(b.bc);
    CK(cudaMemcpyAsync(b.Ef, R, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b.Bf, P, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_aos_to_soa(b.Ef, b.x, b.y, b.z, n, s);
    launch_aos_to_soa(b.Bf, b.px, b.py, b.pz, n, s);
    CK(cudaMemcpyAsync(&b.st->Q, q_macro, sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(b.nacc, 0, (size_t)b.bc.n[0] * b.bc.n[1] * b.bc.n[2] * 2 * sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(b.hist, 0, (size_t)b.bc.n[0] * b.bc.n[1] * b.bc.n[2] * sizeof(int), s));
    CK(cudaMemsetAsync(&b.st->gen, 0, sizeof(unsigned), s));
    launch_reduce_state(b, false, s);
    STAGE("reduce_state");
    launch_drift_to_beam(b, false, s);
    STAGE("bounds");
    enqueue_green(c, s);
    STAGE("green");
    launch_deposit(b, s);
    STAGE("deposit");
    launch_assemble_rho(b, s);
    STAGE("assemble");
    launch_convolution(b, kConvSelfField, s);
    STAGE("convolution");
    launch_grad(b, s);
    STAGE("grad");
    launch_gather_fields(b, s);
    STAGE("gather");
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(Ef, b.Ef, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Bf, b.Bf, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(q_macro, &b.st->Q, sizeof(double), cudaMemcpyDeviceToHost, s));
    rc = check_device_err(c);
    c->have_bunch = false;  // the particle buffers now hold a beam-frame bunch
    c->have_solve = (rc == SCGPU_OK);
    return rc;
}

static int check_bins_args(scgpu_ctx* c, const int* bins, int nbins, int last_emitted) {
    if (nbins < 0 || nbins > kMaxBins) return fail(c, SCGPU_ERR_ARG, "nbins must be in [0, 64]");
    if (nbins > 0 && !bins) return fail(c, SCGPU_ERR_ARG, "null bins");
    if (last_emitted < 0) return fail(c, SCGPU_ERR_ARG, "last_emitted must not be negative");
    return SCGPU_OK;
}

// Switches the resident bunch to the energy-bin loop (nbins > 0) or back to
// one self-field solve (nbins == 0, Distribution::Rebin).  bins[i] is the
// bin of particle i in the order of the last upload; each step computes the
// fields of bins [0, min(last_emitted, nbins)) and their images.
static int set_bins_impl(scgpu_ctx* c, const int* bins, int nbins, int last_emitted, bool device_ptr) {
    if (!c) return SCGPU_ERR_ARG;
    int rc = check_bins_args(c, bins, nbins, last_emitted);
    if (rc) return rc;
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    CK(cudaSetDevice(c->device));
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    const int nactive = last_emitted < nbins ? last_emitted : nbins;
    if (nbins > 0 && b.periodic_z) return fail(c, SCGPU_ERR_UNSUPPORTED, "energy bins with periodic z");
    if (nbins > 0 && c->xfn) return fail(c, SCGPU_ERR_UNSUPPORTED, "energy bins of a sharded bunch");
    if (nbins != b.nbins || nactive != b.nactive) drop_graphs(c);
    if (nbins == 0) {
        b.nbins = b.nactive = 0;
        const int zero = 0;
        CK(cudaMemcpyAsync(&b.st->binned, &zero, sizeof(int), cudaMemcpyHostToDevice, s));
        CK(cudaStreamSynchronize(s));
        return SCGPU_OK;
    }
    if ((rc = ensure_bins(c, nbins))) return rc;
    const long long n = c->n;
    CK(cudaMemsetAsync(b.nacc_bins, 0, (size_t)c->bins_nbins_alloc * mesh_cells(b) * 2 * sizeof(unsigned long long), s));
    int* host_order = b.bin_alt;
    CK(cudaMemcpyAsync(host_order, bins, (size_t)n * sizeof(int), device_ptr ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                       s));
    launch_bins_by_id(host_order, b.id, b.bin, n, s);
    b.nbins = nbins;
    b.nactive = nactive;
    const int one = 1;
    CK(cudaMemcpyAsync(&b.st->binned, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    return SCGPU_OK;
}

int scgpu_set_energy_bins(scgpu_ctx* c, const int* bins, int nbins, int last_emitted) {
    return set_bins_impl(c, bins, nbins, last_emitted, false);
}

int scgpu_get_bin_gammas(scgpu_ctx* c, double* gamma, long long* count) {
    if (!c || !gamma) return fail(c, SCGPU_ERR_ARG, "null argument");
    DevBunch& b = c->b;
    if (b.nbins <= 0 || !b.bst) return fail(c, SCGPU_ERR_STATE, "no energy bins");
    CK(cudaSetDevice(c->device));
    std::vector<StepState> h(b.nbins);
    CK(cudaMemcpyAsync(h.data(), b.bst, b.nbins * sizeof(StepState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < b.nbins; ++k) {
        gamma[k] = h[k].gammaz;
        if (count) count[k] = h[k].bin_count;
    }
    return SCGPU_OK;
}

int scgpu_compute_self_fields_binned(scgpu_ctx* c, long long n, const double* R, const double* P, const int* bins,
                                     int nbins, int last_emitted, double q_macro, double dT, double* Ef, double* Bf,
                                     double* bin_gamma) {
    if (!c || !R || !P || !Ef || !Bf) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!(dT > 0.0)) return fail(c, SCGPU_ERR_ARG, "dT must be positive");
    int rc = check_bins_args(c, bins, nbins, last_emitted);
    if (rc) return rc;
    if (nbins == 0) return fail(c, SCGPU_ERR_ARG, "nbins must be positive");
    if (c->b.periodic_z) return fail(c, SCGPU_ERR_UNSUPPORTED, "energy bins with periodic z");
    if (c->xfn) return fail(c, SCGPU_ERR_UNSUPPORTED, "energy bins of a sharded bunch");
    CK(cudaSetDevice(c->device));
    if ((rc = ensure_particles(c, n))) return rc;
    if ((rc = ensure_bins(c, nbins))) return rc;
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    drop_graphs(c);
    b.bc.dT = dT;
    if (b.bc.coupling == 0.0) b.bc.coupling = 1.0 / (4 * kPi * 8.854187817e-12);
    if (b.bc.mass == 0.0) b.bc.mass = 0.51099892e-03 * 1.0e9;
    bunch_constants(b.bc);
    CK(cudaMemcpyAsync(b.Ef, R, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b.Bf, P, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    launch_aos_to_soa(b.Ef, b.x, b.y, b.z, n, s);
    launch_aos_to_soa(b.Bf, b.px, b.py, b.pz, n, s);
    CK(cudaMemcpyAsync(b.bin, bins, (size_t)n * sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(b.nacc_bins, 0, (size_t)c->bins_nbins_alloc * mesh_cells(b) * 2 * sizeof(unsigned long long), s));
    CK(cudaMemcpyAsync(&b.st->Q, &q_macro, sizeof(double), cudaMemcpyHostToDevice, s));
    const int one = 1;
    CK(cudaMemcpyAsync(&b.st->binned, &one, sizeof(int), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(&b.st->gen, 0, sizeof(unsigned), s));
    b.nbins = nbins;
    b.nactive = last_emitted < nbins ? last_emitted : nbins;
    launch_reduce_state(b, false, s);
    STAGE("reduce_state");
    launch_drift_to_beam(b, false, s);
    STAGE("bounds");
    enqueue_bins_fields(c, s);
    STAGE("bins");
    launch_gather_fields_bins(b, s);
    STAGE("gather");
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(Ef, b.Ef, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(Bf, b.Bf, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    rc = check_device_err(c);
    if (rc == SCGPU_OK && bin_gamma) rc = scgpu_get_bin_gammas(c, bin_gamma, nullptr);
    const int zero = 0;
    cudaMemcpyAsync(&b.st->binned, &zero, sizeof(int), cudaMemcpyHostToDevice, s);
    cudaStreamSynchronize(s);
    b.nbins = b.nactive = 0;
    c->have_bunch = false;  // the particle buffers now hold a beam-frame bunch
    c->have_solve = false;
    return rc;
}

int scgpu_bunch_upload(scgpu_ctx* c, long long n, const double* R, const double* P, const scgpu_bunch_params* bp) {
    if (!c || !R || !P || !bp) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!(bp->dT > 0.0) || !(bp->mass > 0.0)) return fail(c, SCGPU_ERR_ARG, "dT and mass must be positive");
    CK(cudaSetDevice(c->device));
    // A bunch of the same size keeps the device's slot order (slot s takes
    // host particle id[s]): the cell order of the last reorder stays nearly
    // right for the next steps, and no result depends on the order (every
    // sum over particles is exact).
    const bool keep_order = c->have_bunch && n == c->n;
    int rc = ensure_particles(c, n);
    if (rc) return rc;
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    const bool consts_changed = b.bc.dT != bp->dT || b.bc.mass != bp->mass || b.bc.charge != bp->charge ||
                                b.bc.coupling != bp->coupling || b.bc.bz_ext != bp->bz_ext;
    if (consts_changed) drop_graphs(c);
    b.bc.dT = bp->dT;
    b.bc.mass = bp->mass;
    b.bc.charge = bp->charge;
    b.bc.coupling = bp->coupling;
    b.bc.bz_ext = bp->bz_ext;
    bunch_constants(b.bc);
    StepState h{};
    h.t = bp->t;
    h.path_length = bp->path_length;
    for (int k = 0; k < 3; ++k) {
        h.ref_R[k] = bp->ref_R[k];
        h.ref_P[k] = bp->ref_P[k];
    }
    const double o[3] = {0.0, 0.0, 0.0}, q[4] = {1.0, 0.0, 0.0, 0.0};
    trafo_make(h.ref_to_lab, o, q);
    h.Q = bp->q_macro;
    h.step = 0;
    h.gen = 0;
    h.binned = 0;  // energy bins refer to the previous particle order: set them again after an upload
    if (b.nbins > 0) {
        drop_graphs(c);
        b.nbins = b.nactive = 0;
    }
    CK(cudaMemcpyAsync(b.st, &h, sizeof(StepState), cudaMemcpyHostToDevice, s));
    CK(cudaMemsetAsync(b.nacc, 0, (size_t)b.bc.n[0] * b.bc.n[1] * b.bc.n[2] * 2 * sizeof(unsigned long long), s));
    CK(cudaMemsetAsync(b.hist, 0, (size_t)b.bc.n[0] * b.bc.n[1] * b.bc.n[2] * sizeof(int), s));
    CK(cudaMemcpyAsync(b.Ef, R, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b.Bf, P, 3 * n * sizeof(double), cudaMemcpyHostToDevice, s));
    if (keep_order) {
        launch_aos_to_soa_by_id(b.Ef, b.id, b.x, b.y, b.z, n, s);
        launch_aos_to_soa_by_id(b.Bf, b.id, b.px, b.py, b.pz, n, s);
    } else {
        launch_aos_to_soa(b.Ef, b.x, b.y, b.z, n, s);
        launch_aos_to_soa(b.Bf, b.px, b.py, b.pz, n, s);
        launch_iota(b.id, n, s);
        c->steps_done = 0;
    }
    enqueue_psum(c, true, s);
    CK(cudaGetLastError());
    rc = exchange_status(c);
    if (rc == SCGPU_OK) rc = check_device_err(c);
    c->have_bunch = (rc == SCGPU_OK);
    return rc;
}

int scgpu_bunch_download(scgpu_ctx* c, double* R, double* P) {
    if (!c || !R || !P) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    CK(cudaSetDevice(c->device));
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    const long long n = c->n;
    launch_soa_to_aos_by_id(b.x, b.y, b.z, b.id, b.Ef, n, s);
    launch_soa_to_aos_by_id(b.px, b.py, b.pz, b.id, b.Bf, n, s);
    CK(cudaMemcpyAsync(R, b.Ef, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(P, b.Bf, 3 * n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return SCGPU_OK;
}

int scgpu_track(scgpu_ctx* c, int nsteps, double* stats) {
    if (!c || nsteps < 0) return fail(c, SCGPU_ERR_ARG, "bad argument");
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    CK(cudaSetDevice(c->device));
    const bool want = stats != nullptr;
    cudaStream_t s = c->stream;
    CK(cudaEventRecord(c->ev_t0, s));
    for (int k = 0; k < nsteps; ++k) {
        const bool reorder = c->reorder_every > 0 && (c->steps_done % c->reorder_every) == 0;
        if (c->use_graphs && (!c->xfn || c->xcapturable)) {
            cudaGraphExec_t& gx = (c->b.nbins > 0 ? c->graphs_bins : c->graphs)[want ? 1 : 0][reorder ? 1 : 0];
            if (!gx) {
                int rc = build_graph(c, want, reorder, &gx);
                if (rc) return rc;
            }
            CK(cudaGraphLaunch(gx, s));
            c->kernels_launched += (c->b.nbins > 0 ? c->graph_kernels_bins : c->graph_kernels)[want ? 1 : 0][reorder ? 1 : 0];
        } else {
            enqueue_any_step(c, want, reorder, s);
            c->kernels_uncounted = true;
        }
        ++c->steps_done;
        if (want)
            CK(cudaMemcpyAsync(stats + (size_t)k * SCGPU_NSTATS, c->b.st->moments, SCGPU_NSTATS * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
    }
    CK(cudaEventRecord(c->ev_t1, s));
    CK(cudaGetLastError());
    int rc = exchange_status(c);
    if (rc == SCGPU_OK) rc = check_device_err(c);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev_t0, c->ev_t1);
    c->last_ms = ms;
    c->have_solve = (rc == SCGPU_OK && nsteps > 0);
    return rc;
}

int scgpu_get_tracker_state(scgpu_ctx* c, scgpu_tracker_state* out) {
    if (!c || !out) return fail(c, SCGPU_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    StepState h;
    CK(cudaMemcpyAsync(&h, c->b.st, sizeof(StepState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out->t = h.t;
    out->path_length = h.path_length;
    for (int k = 0; k < 3; ++k) {
        out->ref_R[k] = h.ref_R[k];
        out->ref_P[k] = h.ref_P[k];
        out->ref_to_lab_origin[k] = h.ref_to_lab.origin[k];
    }
    for (int k = 0; k < 4; ++k) out->ref_to_lab_quat[k] = h.ref_to_lab.quat[k];
    out->q_macro = h.Q;
    out->step = h.step;
    return SCGPU_OK;
}

int scgpu_beam_parameters(scgpu_ctx* c, scgpu_beam_params* out) {
    if (!c || !out) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    CK(cudaSetDevice(c->device));
    enqueue_stats(c, c->stream);
    double rec[SCGPU_NSTATS];
    CK(cudaMemcpyAsync(rec, c->b.st->moments, sizeof(rec), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    int rc = exchange_status(c);
    if (rc) return rc;
    return scgpu_beam_parameters_from_stats(rec, c->b.bc.Ntot, out);
}

// One row of DataSink::doWriteStatData (DataSink.cpp:281-449) for the resident
// bunch: calcBeamParameters (PartBunchBase.hpp:1529-1614) with calcEMean
// (:2099-2114), get_bounds, the tracker state and particle 0.
int scgpu_stat_row(scgpu_ctx* c, double* row) {
    if (!c || !row) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    CK(cudaSetDevice(c->device));
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    enqueue_stats(c, s);
    double* scratch = b.Ef;  // 3 N doubles >= 12
    launch_bounds(b, scratch, s);
    if (c->xfn) exchange(c, scratch, 6, SCGPU_EXCHANGE_MIN_F64, s);
    launch_find_id(b, 0u, scratch + 6, s);
    double rec[SCGPU_NSTATS], ext[12];
    StepState h;
    CK(cudaMemcpyAsync(rec, b.st->moments, sizeof(rec), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(ext, scratch, sizeof(ext), cudaMemcpyDeviceToHost, s));
    CK(cudaMemcpyAsync(&h, b.st, sizeof(StepState), cudaMemcpyDeviceToHost, s));
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(s));
    int rc = exchange_status(c);
    if (rc) return rc;
    const long long n = b.bc.Ntot;
    const double N = (double)n;
    scgpu_beam_params bp;
    std::memset(&bp, 0, sizeof bp);
    beam_params_from_sums(rec, rec[27], N, &bp);
    // calcEMean: sum of sqrt(P.P + 1) minus N, times m [MeV], over N
    double eKin = rec[27];
    eKin -= N;
    eKin *= b.bc.mass * 1.0e-6;
    eKin /= N;
    // getCharge: sum(Q) over the particles, in storage order
    double Q = 0.0;
    for (long long i = 0; i < n; ++i) Q += h.Q;
    const double m0 = b.bc.mass * 1.E-6;
    const double tmp = 1.0 / std::pow(eKin / m0 + 1., 2.0);
    const double dE = bp.prms[2] * m0 * std::sqrt(1.0 - tmp);
    int k = 0;
    row[k++] = h.t * 1e9;
    row[k++] = h.path_length;
    row[k++] = N;
    row[k++] = Q;
    row[k++] = eKin;
    for (int d = 0; d < 3; ++d) row[k++] = bp.rrms[d];
    for (int d = 0; d < 3; ++d) row[k++] = bp.prms[d];
    for (int d = 0; d < 3; ++d) row[k++] = bp.eps_norm[d];
    for (int d = 0; d < 3; ++d) row[k++] = bp.rmean[d];
    for (int d = 0; d < 3; ++d) row[k++] = h.ref_R[d];
    for (int d = 0; d < 3; ++d) row[k++] = h.ref_P[d];
    for (int d = 0; d < 3; ++d) row[k++] = -ext[3 + d];  // get_maxExtent = rmax
    for (int d = 0; d < 3; ++d) row[k++] = bp.rprms[d];
    row[k++] = rec[mom_idx(0, 5)] / N;  // Dx
    row[k++] = rec[mom_idx(1, 5)] / N;  // DDx
    row[k++] = rec[mom_idx(2, 5)] / N;  // Dy
    row[k++] = rec[mom_idx(3, 5)] / N;  // DDy
    // external B [T] and E [MV/m] at the reference particle: the uniform solenoid field
    row[k++] = 0.0;
    row[k++] = 0.0;
    row[k++] = b.bc.bz_ext;
    row[k++] = 0.0;
    row[k++] = 0.0;
    row[k++] = 0.0;
    row[k++] = dE;
    row[k++] = b.bc.dT * 1e9;
    row[k++] = 0.0;  // outside n sigma: Options::beamHaloBoundary is 0 by default
    for (int d = 0; d < 6; ++d) row[k++] = ext[6 + d];
    return SCGPU_OK;
}

int scgpu_beam_parameters_from_stats(const double* rec, long long n, scgpu_beam_params* out) {
    if (!rec || !out || n <= 0) return SCGPU_ERR_ARG;
    std::memset(out, 0, sizeof(*out));
    beam_params_from_sums(rec, rec[27], (double)n, out);
    return SCGPU_OK;
}

int scgpu_get_field(scgpu_ctx* c, int which, double* out) {
    if (!c || !out) return fail(c, SCGPU_ERR_ARG, "null argument");
    if (!c->have_solve) return fail(c, SCGPU_ERR_STATE, "no self-field solve has run");
    CK(cudaSetDevice(c->device));
    DevBunch& b = c->b;
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    const bool f64 = b.precision == SCGPU_PLAIN_FP64;
    const size_t rs = f64 ? sizeof(double) : sizeof(float);
    if (which == SCGPU_FIELD_PHI) {
        CK(cudaMemcpyAsync(out, b.phi, M * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return SCGPU_OK;
    }
    if (which == SCGPU_FIELD_RHO) {
        std::vector<unsigned char> h(M * rs);
        CK(cudaMemcpyAsync(h.data(), b.rho, M * rs, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (long long i = 0; i < M; ++i)
            out[i] = f64 ? ((const double*)h.data())[i] : (double)((const float*)h.data())[i];
        return SCGPU_OK;
    }
    if (which == SCGPU_FIELD_E) {
        std::vector<unsigned char> h(4 * M * rs);
        CK(cudaMemcpyAsync(h.data(), b.E4, 4 * M * rs, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (long long i = 0; i < M; ++i)
            for (int k = 0; k < 3; ++k)
                out[3 * i + k] = f64 ? ((const double*)h.data())[4 * i + k] : (double)((const float*)h.data())[4 * i + k];
        return SCGPU_OK;
    }
    return fail(c, SCGPU_ERR_ARG, "unknown field");
}

int scgpu_get_mesh(scgpu_ctx* c, scgpu_mesh* out) {
    if (!c || !out) return fail(c, SCGPU_ERR_ARG, "null argument");
    CK(cudaSetDevice(c->device));
    StepState h;
    CK(cudaMemcpyAsync(&h, c->b.st, sizeof(StepState), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int k = 0; k < 3; ++k) {
        out->hr[k] = h.hr[k];
        out->origin[k] = h.origin[k];
        out->rmin[k] = h.mesh_rmin[k];
        out->rmax[k] = h.mesh_rmax[k];
        out->hr_scaled[k] = h.hr_scaled[k];
    }
    out->gammaz = h.gammaz;
    return SCGPU_OK;
}

double scgpu_last_track_ms(const scgpu_ctx* c) { return c ? c->last_ms : 0.0; }

int scgpu_profile_track(scgpu_ctx* c, int nsteps, double* phase_ms) {
    if (!c || nsteps < 0 || !phase_ms) return fail(c, SCGPU_ERR_ARG, "bad argument");
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    if (c->b.nbins > 0) return fail(c, SCGPU_ERR_UNSUPPORTED, "phase profile of a step with energy bins");
    if (c->xfn) return fail(c, SCGPU_ERR_UNSUPPORTED, "phase profile of a sharded bunch");
    CK(cudaSetDevice(c->device));
    DevBunch& b = c->b;
    cudaStream_t s = c->stream;
    cudaEvent_t ev[SCGPU_NPHASES + 1];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int p = 0; p < SCGPU_NPHASES; ++p) phase_ms[p] = 0.0;
    int rc = SCGPU_OK;
    for (int k = 0; k < nsteps && rc == SCGPU_OK; ++k) {
        cudaEventRecord(ev[0], s);
        launch_drift_to_beam(b, true, s, b.precision != SCGPU_PLAIN_FP64);
        launch_advance_reference(b, s);
        cudaEventRecord(ev[1], s);
        launch_deposit(b, s);
        cudaEventRecord(ev[2], s);
        launch_assemble_rho(b, s);
        cudaEventRecord(ev[3], s);
        // the reorder sorts beam-frame positions: it runs where the step runs it
        if (c->reorder_every > 0 && (c->steps_done % c->reorder_every) == 0) enqueue_reorder(c, s);
        ++c->steps_done;
        cudaEventRecord(ev[4], s);
        enqueue_green(c, s);
        cudaEventRecord(ev[5], s);
        launch_convolution(b, kConvSelfField, s);
        cudaEventRecord(ev[6], s);
        launch_grad(b, s);
        cudaEventRecord(ev[7], s);
        launch_gather_kick_push(b, false, s);
        cudaEventRecord(ev[8], s);
        cudaError_t e = cudaEventSynchronize(ev[8]);
        if (e != cudaSuccess) {
            rc = cuda_fail(c, e, "profile step");
            break;
        }
        // event interval i -> phase index (the reorder runs between assemble and green)
        static const int phase_of_interval[SCGPU_NPHASES] = {
            SCGPU_PHASE_DRIFT_BOUNDS, SCGPU_PHASE_DEPOSIT, SCGPU_PHASE_ASSEMBLE,    SCGPU_PHASE_REORDER,
            SCGPU_PHASE_GREEN,        SCGPU_PHASE_CONVOLUTION, SCGPU_PHASE_GRAD, SCGPU_PHASE_GATHER_KICK};
        for (int p = 0; p < SCGPU_NPHASES; ++p) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[p], ev[p + 1]);
            phase_ms[phase_of_interval[p]] += ms;
        }
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (rc) return rc;
    CK(cudaGetLastError());
    return check_device_err(c);
}

int scgpu_kernels_per_step(scgpu_ctx* c) {
    if (!c) return SCGPU_ERR_ARG;
    if (!c->have_bunch) return fail(c, SCGPU_ERR_STATE, "no bunch on the device");
    if (c->xfn && !c->xcapturable) return fail(c, SCGPU_ERR_UNSUPPORTED, "step of a shard with a host exchange");
    CK(cudaSetDevice(c->device));
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(c->own, cudaStreamCaptureModeThreadLocal));
    enqueue_any_step(c, false, false, c->own);
    CK(cudaStreamEndCapture(c->own, &g));
    const int kernels = graph_kernel_nodes(g);
    cudaGraphDestroy(g);
    return kernels;
}

// Kernels launched by scgpu_track on this context so far (reorder and
// statistics steps included), counted from the nodes of the step graphs.
int scgpu_launch_count(scgpu_ctx* c, long long* kernels) {
    if (!c || !kernels) return fail(c, SCGPU_ERR_ARG, "bad argument");
    if (c->kernels_uncounted) return fail(c, SCGPU_ERR_UNSUPPORTED, "steps ran outside step graphs");
    *kernels = c->kernels_launched;
    return SCGPU_OK;
}

}  // extern "C"
