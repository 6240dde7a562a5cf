// sc_batch.cu -- many bunches stepping together (include/scgpu.h, "batches").
//
// Each bunch keeps its own context (buffers, StepState, constants).  A
// batched step launches every kernel of the step once for all bunches: a
// launch carries one item per bunch (bunch, first block, blocks in x and y),
// each block finds its bunch by a binary search over the items, and a device
// copy of each bunch's DevBunch gives the kernel its buffers and sizes.  FFT
// passes are grouped by the transform length of their axis, since the length
// is a template constant of the kernels.  The step order is the single-bunch one (sc_api.cu enqueue_step):
//
//   ref:  reference-particle updates (joined before the gather)
//   main: drift -> deposit -> assemble [-> cell reorder] -> FFT A, B
//   side: Green's function (antiderivative, 8-corner G, three DCT passes)
//   main: (join side) FFT C, D, E -> grad -> (join ref) gather/kick/push
//
// With unchanged membership the step is captured once per variant (with and
// without the periodic cell reorder) and replayed as one graph launch.
#include <algorithm>
#include <cstdio>
#include <map>
#include <string>
#include <vector>

#include "sc_ctx.h"

using namespace sc;

namespace {

constexpr int kCellGridCap = 148 * 16;

__global__ void k_collect_flags(const DevBunch* __restrict__ tab, int n, int* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        out[i] = tab[i].st->err;
        tab[i].st->err = 0;
    }
}

int blocks_for(long long work, int threads, int cap) {
    long long g = (work + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

struct Launch {
    int lane;   // 0 drift, 1 Green's-function branch, 2 deposit, 6 forward FFT, 3 rest of the solve,
                // 4 reference-particle branch, 5 gather (see enqueue_step)
    int kind;   // kBatch* for particle / grid kernels, -1 for an FFT pass
    int pass;   // kPass* when kind == -1
    int L;      // transform length of the pass's axis
    int off;    // first item (one per bunch of the launch)
    int nitems; // bunches of the launch
    int nblocks;
};

}  // namespace

struct scgpu_batch {
    int device = 0;
    int precision = SCGPU_PLAIN_FP64;
    std::vector<scgpu_ctx*> slots;
    std::vector<int> members;   // occupied slots in table order
    cudaStream_t stream = nullptr, side = nullptr, ref = nullptr;
    cudaEvent_t ev_start = nullptr, ev_ref = nullptr;
    // Uploads and downloads of the bunches run here, at the highest stream
    // priority, so that a bunch joining during a long batched round gets SMs
    // as soon as blocks of the round retire instead of waiting for the round.
    cudaStream_t xfer = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_t0 = nullptr, ev_t1 = nullptr;
    std::string err;
    DevBunch* d_tab = nullptr;
    int tab_cap = 0;
    int4* d_work = nullptr;
    size_t work_cap = 0;
    int* d_flags = nullptr;
    std::vector<Launch> launches;
    bool dirty = true;
    // After a membership or tuning change the steps of one track call run
    // without a graph: capturing and instantiating costs more than the few
    // steps a serving round replays.  The next call with the same membership
    // captures (the eager steps have also raised the kernels' shared-memory
    // limits outside any capture).
    bool eager_call = true;
    cudaGraphExec_t graphs[2] = {nullptr, nullptr};  // [reorder]
    long long steps = 0;
    int reorder_every = 16;
    int dep_threads = 256;
    std::map<int, int> fft_variant;  // transform length -> tile-shape variant
    double last_ms = 0.0;
    int in_flight = 0;  // steps launched and not yet waited for
    // Contexts of removed bunches, kept with their device buffers for the
    // next bunch on the same mesh: a serving loop then allocates and frees
    // nothing in steady state (cudaMalloc / cudaFree synchronise the device).
    std::vector<scgpu_ctx*> pool;
    size_t pool_max = 4096;
};

namespace {

int bfail(scgpu_batch* b, int code, const std::string& what) {
    if (b) b->err = what;
    return code;
}

#define BCK(call)                                                                                    \
    do {                                                                                             \
        cudaError_t e_ = (call);                                                                     \
        if (e_ != cudaSuccess) return bfail(b, SCGPU_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void drop_graphs(scgpu_batch* b) {
    for (auto& g : b->graphs) {
        if (g) cudaGraphExecDestroy(g);
        g = nullptr;
    }
}

// the tuned variant of a length, else the line transforms where they exist
int variant_of(const scgpu_batch* b, int L) {
    auto it = b->fft_variant.find(L);
    if (it != b->fft_variant.end()) return it->second;
    return (fft_register_lines() && (L == 64 || L == 128 || L == 256)) ? kFftLinesVariant : 0;
}

// Work tables and launch list of the current membership, uploaded to the device.
int rebuild(scgpu_batch* b) {
    // the tables are rewritten below: nothing enqueued may still read them
    BCK(cudaStreamSynchronize(b->stream));
    BCK(cudaStreamSynchronize(b->side));
    BCK(cudaStreamSynchronize(b->ref));
    drop_graphs(b);
    b->members.clear();
    for (int s = 0; s < (int)b->slots.size(); ++s)
        if (b->slots[s]) b->members.push_back(s);
    const int nm = (int)b->members.size();
    std::vector<DevBunch> tab(nm);
    for (int i = 0; i < nm; ++i) {
        tab[i] = b->slots[b->members[i]]->b;
        // the batched gather has no external-field variant; a sharded bunch needs its exchanges
        if (tab[i].bc.nsol > 0 || tab[i].bc.sharded)
            return bfail(b, SCGPU_ERR_UNSUPPORTED, "beamline elements or a sharded bunch in a batch");
    }
    std::vector<int4> work;
    b->launches.clear();
    auto add_per_bunch = [&](int lane, int kind, auto blocks_of) {
        Launch l{lane, kind, 0, 0, (int)work.size(), 0, 0};
        for (int i = 0; i < nm; ++i) {
            const int nb = blocks_of(tab[i]);
            work.push_back(make_int4(i, l.nblocks, nb, 1));
            l.nblocks += nb;
        }
        l.nitems = (int)work.size() - l.off;
        b->launches.push_back(l);
    };
    auto add_pass = [&](int lane, int pass) {
        std::map<int, std::vector<int>> by_len;
        for (int i = 0; i < nm; ++i) by_len[fft_pass_length(pass, tab[i])].push_back(i);
        for (auto& kv : by_len) {
            Launch l{lane, -1, pass, kv.first, (int)work.size(), 0, 0};
            const int v = variant_of(b, kv.first);
            for (int i : kv.second) {
                int gx = 0, gy = 0;
                fft_pass_grid(pass, tab[i], v, &gx, &gy);
                work.push_back(make_int4(i, l.nblocks, gx, gy));
                l.nblocks += gx * gy;
            }
            l.nitems = (int)work.size() - l.off;
            b->launches.push_back(l);
        }
    };
    auto cells = [](const DevBunch& d) { return (long long)d.bc.n[0] * d.bc.n[1] * d.bc.n[2]; };
    const int dep = b->dep_threads;
    add_per_bunch(0, kBatchDrift, [](const DevBunch& d) { return d.red_blocks; });
    add_per_bunch(1, kBatchIgfTmp, [](const DevBunch& d) {
        return blocks_for((long long)(d.bc.n[0] + 2) * (d.bc.n[1] + 2) * (d.bc.n[2] + 2), 256, kCellGridCap);
    });
    // G is formed from the antiderivative inside the z cosine transforms
    add_pass(1, kPassDctZ);
    add_pass(1, kPassDctY);
    add_pass(1, kPassDctX);
    add_per_bunch(2, kBatchDeposit, [dep](const DevBunch& d) { return blocks_for(d.bc.N, dep, 148 * 8 * 256 / dep); });
    add_per_bunch(2, kBatchAssemble, [&](const DevBunch& d) { return blocks_for(cells(d), 256, kCellGridCap); });
    add_per_bunch(4, kBatchAdvance, [](const DevBunch&) { return 1; });
    add_pass(6, kPassZR2C);
    add_pass(6, kPassYFwd);
    add_pass(3, kPassXConv);
    add_pass(3, kPassYInv);
    add_pass(3, kPassZC2R);
    add_per_bunch(3, kBatchGrad, [&](const DevBunch& d) { return blocks_for(cells(d), 256, kCellGridCap); });
    add_per_bunch(5, kBatchGather, [](const DevBunch& d) { return d.red_blocks; });
    if (nm > b->tab_cap) {
        if (b->d_tab) cudaFree(b->d_tab);
        if (b->d_flags) cudaFree(b->d_flags);
        b->d_tab = nullptr;
        b->d_flags = nullptr;
        const int cap = std::max(nm, 2 * b->tab_cap);
        BCK(cudaMalloc(&b->d_tab, (size_t)cap * sizeof(DevBunch)));
        BCK(cudaMalloc(&b->d_flags, (size_t)cap * sizeof(int)));
        b->tab_cap = cap;
    }
    if (work.size() > b->work_cap) {
        if (b->d_work) cudaFree(b->d_work);
        b->d_work = nullptr;
        const size_t cap = std::max(work.size(), 2 * b->work_cap);
        BCK(cudaMalloc(&b->d_work, cap * sizeof(int4)));
        b->work_cap = cap;
    }
    if (nm) BCK(cudaMemcpy(b->d_tab, tab.data(), (size_t)nm * sizeof(DevBunch), cudaMemcpyHostToDevice));
    if (!work.empty()) BCK(cudaMemcpy(b->d_work, work.data(), work.size() * sizeof(int4), cudaMemcpyHostToDevice));
    b->dirty = false;
    b->eager_call = true;
    return SCGPU_OK;
}

void enqueue_lane(scgpu_batch* b, int lane, cudaStream_t s) {
    for (const Launch& l : b->launches) {
        if (l.lane != lane) continue;
        const int4* w = b->d_work + l.off;
        if (l.kind < 0)
            launch_fft_pass_batch(l.pass, l.L, b->precision, variant_of(b, l.L), b->d_tab, w, l.nitems, l.nblocks, s);
        else
            launch_batch(l.kind, b->precision, b->dep_threads, b->d_tab, w, l.nitems, l.nblocks, s);
    }
}

void enqueue_step(scgpu_batch* b, bool reorder) {
    cudaStream_t s = b->stream;
    cudaEventRecord(b->ev_start, s);
    cudaStreamWaitEvent(b->ref, b->ev_start, 0);
    enqueue_lane(b, 4, b->ref);  // reference particles
    cudaEventRecord(b->ev_ref, b->ref);
    enqueue_lane(b, 0, s);       // drift
    cudaEventRecord(b->ev_fork, s);
    cudaStreamWaitEvent(b->side, b->ev_fork, 0);
    enqueue_lane(b, 1, b->side);  // Green's functions
    cudaEventRecord(b->ev_join, b->side);
    enqueue_lane(b, 2, s);       // deposit, assemble
    if (reorder)
        for (int m : b->members) ctx_enqueue_reorder(b->slots[m], s);
    enqueue_lane(b, 6, s);       // FFT A, B
    cudaStreamWaitEvent(s, b->ev_join, 0);
    enqueue_lane(b, 3, s);       // FFT C, D, E, grad
    cudaStreamWaitEvent(s, b->ev_ref, 0);
    enqueue_lane(b, 5, s);       // gather, kick, push
}

int check_flags(scgpu_batch* b) {
    const int nm = (int)b->members.size();
    if (!nm) return SCGPU_OK;
    k_collect_flags<<<(nm + 127) / 128, 128, 0, b->stream>>>(b->d_tab, nm, b->d_flags);
    std::vector<int> h(nm);
    BCK(cudaMemcpyAsync(h.data(), b->d_flags, nm * sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    BCK(cudaStreamSynchronize(b->stream));
    for (int i = 0; i < nm; ++i)
        if (h[i]) {
            scgpu_ctx* c = b->slots[b->members[i]];
            const int rc = ctx_status_from_flags(c, h[i]);
            return bfail(b, rc, "slot " + std::to_string(b->members[i]) + ": " + c->err);
        }
    return SCGPU_OK;
}

// Enqueues nsteps batched steps on the batch stream and returns.
int launch(scgpu_batch* b, int nsteps) {
    BCK(cudaSetDevice(b->device));
    if (b->dirty) {
        int rc = rebuild(b);
        if (rc) return rc;
    }
    b->in_flight = nsteps;
    if (b->members.empty()) return SCGPU_OK;
    BCK(cudaEventRecord(b->ev_t0, b->stream));
    for (int k = 0; k < nsteps; ++k) {
        const bool reorder = b->reorder_every > 0 && (b->steps % b->reorder_every) == 0;
        cudaGraphExec_t& gx = b->graphs[reorder ? 1 : 0];
        if (!gx && !b->eager_call) {
            cudaGraph_t g = nullptr;
            BCK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            enqueue_step(b, reorder);
            cudaError_t e = cudaStreamEndCapture(b->stream, &g);
            if (e != cudaSuccess) return bfail(b, SCGPU_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&gx, g, cudaGraphInstantiateFlagUseNodePriority);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return bfail(b, SCGPU_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        }
        if (gx)
            BCK(cudaGraphLaunch(gx, b->stream));
        else
            enqueue_step(b, reorder);
        ++b->steps;
    }
    BCK(cudaEventRecord(b->ev_t1, b->stream));
    BCK(cudaGetLastError());
    b->eager_call = false;
    return SCGPU_OK;
}

// Waits for the launched steps; device error flags become the status.
int wait(scgpu_batch* b) {
    BCK(cudaSetDevice(b->device));
    const int nsteps = b->in_flight;
    b->in_flight = 0;
    if (b->members.empty()) {
        b->last_ms = 0.0;
        return SCGPU_OK;
    }
    int rc = check_flags(b);
    float ms = 0.f;
    if (nsteps > 0) cudaEventElapsedTime(&ms, b->ev_t0, b->ev_t1);
    b->last_ms = ms;
    for (int m : b->members) b->slots[m]->have_solve = (rc == SCGPU_OK && nsteps > 0);
    return rc;
}

int track(scgpu_batch* b, int nsteps) {
    int rc = launch(b, nsteps);
    if (rc) return rc;
    return wait(b);
}

// A parked context for a new bunch on the same mesh, taken out of the pool:
// the smallest one with enough particle capacity, else the largest (its
// particle arrays then grow on upload; the grids are reused either way);
// null if no parked context has this mesh.
scgpu_ctx* take_pooled(scgpu_batch* b, const scgpu_solver_params& q, long long n) {
    int best = -1;
    for (int i = 0; i < (int)b->pool.size(); ++i) {
        const scgpu_ctx* c = b->pool[i];
        if (c->sp.mx != q.mx || c->sp.my != q.my || c->sp.mt != q.mt || c->sp.bboxincr != q.bboxincr) continue;
        if (best < 0) {
            best = i;
            continue;
        }
        const long long cb = b->pool[best]->capacity, ci = c->capacity;
        const bool fits_b = cb >= n, fits_i = ci >= n;
        if ((fits_i && (!fits_b || ci < cb)) || (!fits_i && !fits_b && ci > cb)) best = i;
    }
    if (best < 0) return nullptr;
    scgpu_ctx* c = b->pool[best];
    b->pool.erase(b->pool.begin() + best);
    return c;
}

void drain_pool(scgpu_batch* b) {
    for (scgpu_ctx* c : b->pool) scgpu_destroy(c);
    b->pool.clear();
}

}  // namespace

extern "C" {

int scgpu_batch_create(scgpu_batch** out, int device, int precision) {
    if (!out) return SCGPU_ERR_ARG;
    *out = nullptr;
    if (precision != SCGPU_PLAIN_FP64 && precision != SCGPU_MIXED) return SCGPU_ERR_ARG;
    if (cudaSetDevice(device) != cudaSuccess) return SCGPU_ERR_CUDA;
    scgpu_batch* b = new scgpu_batch();
    b->device = device;
    b->precision = precision;
    int least = 0, greatest = 0;
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    if (cudaStreamCreateWithPriority(&b->xfer, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        // the main chain at the highest priority, the Green's functions at the
        // lowest (kept in the step graphs: cudaGraphInstantiateFlagUseNodePriority)
        cudaStreamCreateWithPriority(&b->stream, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, least) != cudaSuccess ||
        cudaStreamCreateWithPriority(&b->ref, cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_start, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_ref, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreate(&b->ev_t0) != cudaSuccess || cudaEventCreate(&b->ev_t1) != cudaSuccess) {
        scgpu_batch_destroy(b);
        return SCGPU_ERR_CUDA;
    }
    *out = b;
    return SCGPU_OK;
}

void scgpu_batch_destroy(scgpu_batch* b) {
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    drop_graphs(b);
    drain_pool(b);
    for (scgpu_ctx*& c : b->slots)
        if (c) {
            scgpu_destroy(c);
            c = nullptr;
        }
    if (b->d_tab) cudaFree(b->d_tab);
    if (b->d_work) cudaFree(b->d_work);
    if (b->d_flags) cudaFree(b->d_flags);
    for (cudaEvent_t e : {b->ev_fork, b->ev_join, b->ev_t0, b->ev_t1, b->ev_start, b->ev_ref})
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->xfer) cudaStreamDestroy(b->xfer);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->ref) cudaStreamDestroy(b->ref);
    delete b;
}

const char* scgpu_batch_last_error(const scgpu_batch* b) { return b ? b->err.c_str() : "null batch"; }

int scgpu_batch_add(scgpu_batch* b, const scgpu_solver_params* p, long long n, const double* R, const double* P,
                    const scgpu_bunch_params* bp) {
    if (!b || !p || !R || !P || !bp) return bfail(b, SCGPU_ERR_ARG, "null argument");
    scgpu_solver_params q = *p;
    q.precision = b->precision;
    scgpu_ctx* c = take_pooled(b, q, n);
    int rc = SCGPU_OK;
    if (!c) {
        rc = scgpu_create(&c, &q, b->device);
        if (rc == SCGPU_ERR_OOM && !b->pool.empty()) {
            // parked contexts hold the memory: release them and try once more
            drain_pool(b);
            rc = scgpu_create(&c, &q, b->device);
        }
        if (rc) return bfail(b, rc, "scgpu_create failed for the new bunch");
        scgpu_set_stream(c, b->xfer);
    }
    rc = scgpu_bunch_upload(c, n, R, P, bp);
    if (rc == SCGPU_ERR_OOM && !b->pool.empty()) {
        drain_pool(b);
        rc = scgpu_bunch_upload(c, n, R, P, bp);
    }
    if (rc) {
        b->err = scgpu_last_error(c);
        scgpu_destroy(c);
        return rc;
    }
    int slot = -1;
    for (int s = 0; s < (int)b->slots.size(); ++s)
        if (!b->slots[s]) {
            slot = s;
            break;
        }
    if (slot < 0) {
        slot = (int)b->slots.size();
        b->slots.push_back(nullptr);
    }
    b->slots[slot] = c;
    b->dirty = true;
    return slot;
}

int scgpu_batch_remove(scgpu_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size() || !b->slots[slot]) return bfail(b, SCGPU_ERR_ARG, "no such slot");
    cudaSetDevice(b->device);
    // steps in flight still read this bunch (and the flag check reads its
    // state): finish them first
    if (b->in_flight) {
        const int rc = wait(b);
        if (rc) return rc;
    }
    cudaStreamSynchronize(b->stream);
    cudaStreamSynchronize(b->side);
    cudaStreamSynchronize(b->ref);
    scgpu_ctx* c = b->slots[slot];
    b->slots[slot] = nullptr;
    b->dirty = true;
    if (b->pool.size() < b->pool_max) {
        c->have_bunch = false;
        c->have_solve = false;
        b->pool.push_back(c);
    } else {
        scgpu_destroy(c);
    }
    return SCGPU_OK;
}

int scgpu_batch_trim(scgpu_batch* b) {
    if (!b) return SCGPU_ERR_ARG;
    cudaSetDevice(b->device);
    drain_pool(b);
    return SCGPU_OK;
}

int scgpu_batch_launch(scgpu_batch* b, int nsteps) {
    if (!b || nsteps < 0) return bfail(b, SCGPU_ERR_ARG, "bad argument");
    if (b->in_flight) return bfail(b, SCGPU_ERR_STATE, "steps are already in flight: call scgpu_batch_wait");
    return launch(b, nsteps);
}

int scgpu_batch_wait(scgpu_batch* b) {
    if (!b) return SCGPU_ERR_ARG;
    return wait(b);
}

int scgpu_batch_done(scgpu_batch* b) {
    if (!b) return SCGPU_ERR_ARG;
    if (!b->in_flight || b->members.empty()) return 1;
    cudaSetDevice(b->device);
    const cudaError_t e = cudaEventQuery(b->ev_t1);
    if (e == cudaSuccess) return 1;
    if (e == cudaErrorNotReady) return 0;
    return bfail(b, SCGPU_ERR_CUDA, std::string("batch_done: ") + cudaGetErrorString(e));
}

scgpu_ctx* scgpu_batch_member(scgpu_batch* b, int slot) {
    if (!b || slot < 0 || slot >= (int)b->slots.size()) return nullptr;
    return b->slots[slot];
}

int scgpu_batch_size(const scgpu_batch* b) {
    if (!b) return 0;
    int k = 0;
    for (scgpu_ctx* c : b->slots) k += c != nullptr;
    return k;
}

int scgpu_batch_track(scgpu_batch* b, int nsteps) {
    if (!b || nsteps < 0) return bfail(b, SCGPU_ERR_ARG, "bad argument");
    if (b->in_flight) {
        const int rc = wait(b);
        if (rc) return rc;
    }
    return track(b, nsteps);
}

double scgpu_batch_last_track_ms(const scgpu_batch* b) { return b ? b->last_ms : 0.0; }

int scgpu_batch_set_tuning(scgpu_batch* b, int deposit_threads, int L, int fft_variant) {
    if (!b) return SCGPU_ERR_ARG;
    if (deposit_threads != 128 && deposit_threads != 256 && deposit_threads != 512)
        return bfail(b, SCGPU_ERR_ARG, "deposit threads must be 128, 256 or 512");
    if (fft_variant < 0 || fft_variant >= kFftVariants) return bfail(b, SCGPU_ERR_ARG, "unknown FFT variant");
    if (deposit_threads != b->dep_threads) b->dirty = true;
    b->dep_threads = deposit_threads;
    if (L > 0 && variant_of(b, L) != fft_variant) {
        b->fft_variant[L] = fft_variant;
        b->dirty = true;
    }
    return SCGPU_OK;
}

int scgpu_batch_get_tuning(const scgpu_batch* b, int L, int* deposit_threads, int* fft_variant) {
    if (!b) return SCGPU_ERR_ARG;
    if (deposit_threads) *deposit_threads = b->dep_threads;
    if (fft_variant) *fft_variant = variant_of(b, L);
    return SCGPU_OK;
}

int scgpu_batch_autotune(scgpu_batch* b, int trial_steps) {
    if (!b || trial_steps < 1) return bfail(b, SCGPU_ERR_ARG, "trial_steps must be >= 1");
    int taken = 0;
    // time one candidate: one step to capture the graph, then trial_steps timed
    auto time_it = [&](double* ms) -> int {
        int rc = track(b, 1);
        if (rc) return rc;
        rc = track(b, trial_steps);
        if (rc) return rc;
        taken += 1 + trial_steps;
        *ms = b->last_ms;
        return SCGPU_OK;
    };
    double best = 0.0;
    int best_dep = b->dep_threads;
    for (int t : {256, 128, 512}) {
        b->dep_threads = t;
        b->dirty = true;
        double ms = 0.0;
        int rc = time_it(&ms);
        if (rc) return rc;
        if (t == 256 || ms < best) {
            best = ms;
            best_dep = t;
        }
    }
    b->dep_threads = best_dep;
    b->dirty = true;
    std::vector<int> lengths;
    for (scgpu_ctx* c : b->slots)
        if (c)
            for (int d = 0; d < 3; ++d) lengths.push_back(2 * c->b.bc.n[d]);
    std::sort(lengths.begin(), lengths.end());
    lengths.erase(std::unique(lengths.begin(), lengths.end()), lengths.end());
    for (int L : lengths) {
        double best_ms = 0.0;
        int best_v = 0;
        for (int v = 0; v < kFftVariants; ++v) {
            double ms = 0.0;
            b->fft_variant[L] = v;
            b->dirty = true;
            int rc = time_it(&ms);
            if (rc) return rc;
            if (v == 0 || ms < best_ms) {
                best_ms = ms;
                best_v = v;
            }
        }
        b->fft_variant[L] = best_v;
        b->dirty = true;
    }
    return taken;
}

}  // extern "C"
