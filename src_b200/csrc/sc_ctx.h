// sc_ctx.h -- the context behind an scgpu_ctx handle, shared by the C ABI
// translation units (sc_api.cu: one bunch; sc_batch.cu: many bunches that
// step together, each held in its own context).
#pragma once

#include <string>
#include <vector>

#include "scgpu.h"
#include "sc_internal.h"

struct scgpu_ctx {
    int device = 0;
    scgpu_solver_params sp{};
    sc::DevBunch b{};
    cudaStream_t stream = nullptr;   // work stream (own or the caller's)
    cudaStream_t own = nullptr;
    cudaStream_t side = nullptr;     // Green's function branch
    cudaStream_t ref = nullptr;      // reference-particle branch
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    cudaEvent_t ev_start = nullptr, ev_ref = nullptr;
    long long capacity = 0;
    long long n = 0;
    bool have_bunch = false;
    bool have_solve = false;
    int digit_bits = 0;
    std::string err;
    double last_ms = 0.0;
    cudaGraphExec_t graphs[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [stats][reorder]
    int graph_kernels[2][2] = {{0, 0}, {0, 0}};       // kernel nodes of each step graph
    int graph_kernels_bins[2][2] = {{0, 0}, {0, 0}};
    long long kernels_launched = 0;   // kernels of the steps scgpu_track launched as graphs
    bool kernels_uncounted = false;   // a step ran outside a graph (host exchange)
    bool use_graphs = true;
    int reorder_every = 32;   // put the particle arrays in cell order every k steps (0: never)
    long long steps_done = 0; // steps since the last upload
    size_t smem_fft = 0;
    // energy bins and image charges (buffers allocated on first use)
    cudaGraphExec_t graphs_bins[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // [stats][reorder]
    long long bin_capacity = 0;
    int bins_nbins_alloc = 0;     // bins the per-bin accumulators were sized for
    void* spec_fwd_buf = nullptr; // plain form: forward spectrum of a bin
    void* ghat_alt = nullptr;     // second spectrum buffers: the side stream builds bin k+1's Green's
    void* ghat_img_alt = nullptr; // functions while the main stream convolves bin k
    double* phi_img_buf = nullptr; // the image's potential of the bin being convolved
    cudaEvent_t ev_bin[sc::kMaxBins] = {};
    cudaEvent_t ev_used[sc::kMaxBins] = {};
    // beamline elements (scgpu_add_solenoid): host copy and device table
    std::vector<sc::MapElem> elements;
    sc::MapElem* d_elements = nullptr;
    std::vector<double*> map_grids;  // device grids of the elements' 2D maps
    // sharded bunch (scgpu_set_exchange): this context holds one rank's shard
    scgpu_exchange_fn xfn = nullptr;
    void* xuser = nullptr;
    long long ntot = 0;        // particles over all ranks
    bool xcapturable = false;
    int xerr = 0;              // first failing exchange of the last enqueue
};

namespace sc {

// Records `what` as the context's last error and returns `code`.
int ctx_fail(scgpu_ctx* c, int code, const std::string& what);
// Counting sort of the particle arrays into cell order (enqueued on s).
void ctx_enqueue_reorder(scgpu_ctx* c, cudaStream_t s);
// Turns a device error flag word into a status code (and clears the flag).
int ctx_status_from_flags(scgpu_ctx* c, int flags);

}  // namespace sc
