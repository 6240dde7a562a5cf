// sc_particles.cu -- particle-side kernels of the space-charge step.
//
// Compiled with -fmad=false: every per-particle expression of the plain form
// rounds like the reference's CPU code (push, kick, frame transforms, CIC
// weights).  Divisions by a per-bunch or per-step constant use div_rcp (a
// correctly rounded quotient from the correctly rounded reciprocal), so they
// stay bit-exact.  The mixed form's particle update (mixed_particle) writes
// its fused multiply-adds explicitly.
//
//   k_reduce_state       momentum sums (+ beam statistics) and the beam frame
//   k_drift_to_beam      half drift, reference -> beam frame, bounds, mesh
//   k_advance_reference  reference particle and frame update (one thread)
//   k_cell_keys          CIC cell key and rank in its cell (counting sort for the reorder)
//   k_deposit            warp groups by cell, exact group sums, exact integer node sums
//   k_assemble_rho       node sums -> charge density on the n^3 cell field
//   k_igf_tmp, k_igf_G   integrated Green's function (FFTPoissonSolver.cpp:459-522)
//   k_grad               -Grad phi (UniformCartesian.hpp:2129-2203), boost scaling
//   k_gather_kick_push   CIC gather, B from E, back to the reference frame, Boris
//                        kick, half drift, reference-frame update, momentum sums
//   k_gather_staged      the same with the particle state streamed through shared
//                        memory by bulk copies (cp.async.bulk, mbarrier), the default
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <unordered_map>

#include "sc_bulk.cuh"
#include "sc_ddmath.cuh"
#include "sc_exact.cuh"
#include "sc_internal.h"

namespace sc {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;

// Per-step constants (mesh, frames) are staged once per block in shared
// memory.  Reading them through fresh() inside a particle loop keeps the
// compiler from hoisting all of them into registers for the whole loop
// (which spills); each value is re-read from shared memory where it is used.
template <typename P>
__device__ __forceinline__ const P* fresh(const P* p) {
    asm volatile("" : "+l"(p));
    return p;
}

// The block a kernel body works on and the number of blocks working on the
// same bunch: blockIdx.x / gridDim.x of a single-bunch launch, or an entry of
// the work table of a batched launch.
struct VB {
    int blk, nblk;
};
__device__ __forceinline__ VB vb_grid() { return VB{(int)blockIdx.x, (int)gridDim.x}; }

struct MeshConsts {
    double hr[3], rhr[3], org[3];
};
__device__ __forceinline__ void load_mesh_consts(MeshConsts& m, const StepState* st) {
    if (threadIdx.x < 3) {
        m.hr[threadIdx.x] = st->hr[threadIdx.x];
        m.rhr[threadIdx.x] = st->rhr[threadIdx.x];
        m.org[threadIdx.x] = st->origin[threadIdx.x];
    }
}

// ------------------------------------------------------------ reductions
// Last-block-done: true in exactly one of the nblk blocks working on a bunch,
// after every block's partials are visible.  The caller resets the ticket.
__device__ __forceinline__ bool last_block(unsigned* ticket, int nblk) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == (unsigned)nblk - 1u);
    __syncthreads();
    return am_last;
}

// Exact block sum of NV fixed-point values per thread into partials[block][NV].
template <int NV>
__device__ __forceinline__ void block_sum_ex(i128 (&v)[NV], i128* __restrict__ partials, int blk) {
    __shared__ i128 sm[NV][kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += ex_shfl_down(v[k], off);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sm[k][warp] = v[k];
    __syncthreads();
    for (int k = threadIdx.x; k < NV; k += blockDim.x) {
        i128 s = 0;
        for (int w = 0; w < kWarps; ++w) s += sm[k][w];
        partials[(size_t)blk * NV + k] = s;
    }
}

// Exact total of column k over nb block partials, rounded once: out[k].
// For a few columns every thread of the (last) block loads a share of the
// rows, so all loads are in flight at once instead of one warp walking each
// column; the integer sums are exact, so the order does not matter.
template <int NV>
__device__ __forceinline__ void final_sum_ex(const i128* partials, int nb, double* out, i128* exact = nullptr) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if constexpr (NV <= 8) {
        i128 s[NV];
#pragma unroll
        for (int k = 0; k < NV; ++k) s[k] = 0;
        for (int b = threadIdx.x; b < nb; b += blockDim.x) {
            const unsigned long long* q = reinterpret_cast<const unsigned long long*>(partials + (size_t)b * NV);
#pragma unroll
            for (int k = 0; k < NV; ++k) s[k] += (i128)(((u128)__ldcg(q + 2 * k + 1) << 64) | __ldcg(q + 2 * k));
        }
        __shared__ i128 sm[NV][kWarps];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
#pragma unroll
            for (int k = 0; k < NV; ++k) s[k] += ex_shfl_down(s[k], off);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < NV; ++k) sm[k][warp] = s[k];
        __syncthreads();
        if (threadIdx.x < NV) {
            i128 t = 0;
            for (int w = 0; w < kWarps; ++w) t += sm[threadIdx.x][w];
            out[threadIdx.x] = ex_to_double(t);
            if (exact) exact[threadIdx.x] = t;
        }
        return;
    }
    for (int k = warp; k < NV; k += kWarps) {
        i128 s = 0;
        for (int b = lane; b < nb; b += 32) {
            const unsigned long long* q = reinterpret_cast<const unsigned long long*>(partials + (size_t)b * NV + k);
            const unsigned long long lo = __ldcg(q), hi = __ldcg(q + 1);
            s += (i128)(((u128)hi << 64) | lo);
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += ex_shfl_down(s, off);
        if (lane == 0) {
            out[k] = ex_to_double(s);
            if (exact) exact[k] = s;
        }
    }
}

// Same pattern with min (exact, order-independent), all threads loading.
template <int NV>
__device__ __forceinline__ void final_min(const double* partials, int nb, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double s[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) s[k] = INFINITY;
    for (int b = threadIdx.x; b < nb; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < NV; ++k) s[k] = fmin(s[k], __ldcg(partials + (size_t)b * NV + k));
    __shared__ double sm[NV][kWarps];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < NV; ++k) s[k] = fmin(s[k], __shfl_down_sync(kFull, s[k], off));
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sm[k][warp] = s[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        double t = INFINITY;
        for (int w = 0; w < kWarps; ++w) t = fmin(t, sm[threadIdx.x][w]);
        out[threadIdx.x] = t;
    }
}

// A 128-bit exact sum as four 32-bit chunks of its two's complement, each
// in a 64-bit word: summing the words of several ranks as integers and
// recombining gives the exact total (mod 2^128, which holds it).
__device__ __forceinline__ void put_limbs(unsigned long long* dst, i128 v) {
#pragma unroll
    for (int j = 0; j < 4; ++j) dst[j] = (unsigned long long)(unsigned)((u128)v >> (32 * j));
}
__device__ __forceinline__ i128 get_limbs(const unsigned long long* src) {
    u128 t = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) t += (u128)src[j] << (32 * j);
    return (i128)t;
}

// moments in OPAL's order (x, px, y, py, z, pz), PartBunchBase.hpp:2185-2259,
// plus sum of gamma (:1588-1593) as value 27.
// Each product is rounded to a double as in the reference; the sums are exact.
__device__ __forceinline__ void accumulate_moments(i128 (&m)[28], const double* R, const double* P) {
    double part[6] = {R[0], P[0], R[1], P[1], R[2], P[2]};
    int l = 6;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        m[i] += ex_from(part[i]);
#pragma unroll
        for (int j = 0; j <= i; ++j) m[l++] += ex_from(part[i] * part[j]);
    }
    m[27] += ex_from(sqrt(1.0 + dot3(P, P)));
}

// ------------------------------------------------------------ state reduction
// STATS: the 27 moment sums and the sum of gamma of the current state, into
// st->moments / st->gsum.  Otherwise the momentum sums into st->psum (and,
// with init_frame, the beam frame of the next step).
template <bool STATS>
__device__ __forceinline__ void reduce_state_body(const BunchConst& bc, const double* __restrict__ x,
                                                  const double* __restrict__ y, const double* __restrict__ z,
                                                  const double* __restrict__ px, const double* __restrict__ py,
                                                  const double* __restrict__ pz, StepState* st, double* partials,
                                                  unsigned* ticket, bool init_frame, VB g) {
    constexpr int NV = STATS ? 28 : 3;
    i128 v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0;
    for (long long i = g.blk * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)g.nblk * blockDim.x) {
        double P[3] = {px[i], py[i], pz[i]};
        if constexpr (STATS) {
            double R[3] = {x[i], y[i], z[i]};
            accumulate_moments(v, R, P);
        } else {
            v[0] += ex_from(P[0]);
            v[1] += ex_from(P[1]);
            v[2] += ex_from(P[2]);
        }
    }
    i128* xpart = reinterpret_cast<i128*>(partials);
    block_sum_ex<NV>(v, xpart, g.blk);
    if (!last_block(ticket, g.nblk)) return;
    __shared__ double tot[NV];
    __shared__ i128 ex[NV];
    final_sum_ex<NV>(xpart, g.nblk, tot, ex);
    __syncthreads();
    if (bc.sharded) {  // this rank's exact sums; k_finish_* completes after the exchange
        for (int k = threadIdx.x; k < NV; k += blockDim.x) put_limbs(st->xlimbs + 4 * k, ex[k]);
        if (threadIdx.x == 0) *ticket = 0u;
        return;
    }
    if (threadIdx.x == 0) {
        if constexpr (STATS) {
            for (int k = 0; k < 27; ++k) st->moments[k] = tot[k];
            st->gsum = tot[27];
        } else {
            st->psum[0] = tot[0];
            st->psum[1] = tot[1];
            st->psum[2] = tot[2];
            if (init_frame && !derive_beam_frame(*st, bc)) atomicOr(&st->err, kFlagFrame);
        }
        *ticket = 0u;
    }
}
template <bool STATS>
__global__ void __launch_bounds__(kThreads) k_reduce_state(BunchConst bc, const double* __restrict__ x,
                                                           const double* __restrict__ y, const double* __restrict__ z,
                                                           const double* __restrict__ px, const double* __restrict__ py,
                                                           const double* __restrict__ pz, StepState* st,
                                                           double* partials, unsigned* ticket, bool init_frame) {
    reduce_state_body<STATS>(bc, x, y, z, px, py, pz, st, partials, ticket, init_frame, vb_grid());
}

// ------------------------------------------------------------ drift + frame
// The mesh of this step from the bounds in s.bmin / s.bmax, and the charge
// of the scatter: Q *= dt; scatter; Q /= dt  (PartBunch.cpp:493-495); the
// energy-bin loop restores Q from its copy after every bin
// (ParallelTTracker.cpp:570-576).
__device__ __forceinline__ void finish_mesh(StepState& s, const BunchConst& bc) {
    if (!derive_mesh(s, bc)) atomicOr(&s.err, kFlagMesh);
    s.qdt = s.Q * bc.dT;
    if (!s.binned) s.Q = s.qdt / bc.dT;
    s.gen += 1u;
    if (s.gen == 0u) s.gen = 1u;
}

__device__ __forceinline__ void bounds_tail(const BunchConst& bc, double (&v)[6], StepState* st, double* partials,
                                            unsigned* ticket, VB g);

// Products and sums of the mixed form's FP64 steps, written as fused
// multiply-adds (this file is compiled without contraction).
__device__ __forceinline__ void matvec_fma(const double* M, const double* v, double* r) {
    const double r0 = fma(M[0], v[0], fma(M[1], v[1], M[2] * v[2]));
    const double r1 = fma(M[3], v[0], fma(M[4], v[1], M[5] * v[2]));
    const double r2 = fma(M[6], v[0], fma(M[7], v[1], M[8] * v[2]));
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
}
__device__ __forceinline__ void cross_fma(const double* a, const double* b, double* r) {
    const double r0 = fma(a[1], b[2], -a[2] * b[1]);
    const double r1 = fma(a[2], b[0], -a[0] * b[2]);
    const double r2 = fma(a[0], b[1], -a[1] * b[0]);
    r[0] = r0;
    r[1] = r1;
    r[2] = r2;
}

// MIXED: the mixed form's half drift R += (c dt / 2) P / gamma and beam-frame
// translation and rotation in fused multiply-adds (the half drift of its
// gather), in place of the reference's unitless round trip.
template <bool DRIFT, bool MIXED = false>
__device__ __forceinline__ void drift_body(const BunchConst& bc, double* __restrict__ x, double* __restrict__ y,
                                           double* __restrict__ z, const double* __restrict__ px,
                                           const double* __restrict__ py, const double* __restrict__ pz, StepState* st,
                                           double* partials, unsigned* ticket, VB g) {
    __shared__ Trafo r2b_s;
    if (threadIdx.x == 0) r2b_s = st->r2b;
    __syncthreads();
    double v[6] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};  // min x,y,z, -max x,y,z
    // The next particle's loads are issued before the current one is
    // computed, so each thread keeps two particles' reads in flight.
    const long long stride = (long long)g.nblk * blockDim.x;
    long long i = g.blk * (long long)blockDim.x + threadIdx.x;
    double Rn[3] = {0.0, 0.0, 0.0}, Pn[3] = {0.0, 0.0, 0.0};
    if (i < bc.N) {
        Rn[0] = x[i], Rn[1] = y[i], Rn[2] = z[i];
        if constexpr (DRIFT) Pn[0] = px[i], Pn[1] = py[i], Pn[2] = pz[i];
    }
    for (; i < bc.N; i += stride) {
        double R[3] = {Rn[0], Rn[1], Rn[2]};
        const double P[3] = {Pn[0], Pn[1], Pn[2]};
        const long long j = i + stride;
        if (j < bc.N) {
            Rn[0] = x[j], Rn[1] = y[j], Rn[2] = z[j];
            if constexpr (DRIFT) Pn[0] = px[j], Pn[1] = py[j], Pn[2] = pz[j];
        }
        if constexpr (DRIFT) {
            double b[3];
            if constexpr (MIXED) {
                const double gm = sqrt(fma(P[0], P[0], fma(P[1], P[1], fma(P[2], P[2], 1.0))));
                const double hv = (0.5 * bc.s_cdt) / gm;
                const Trafo* t = fresh(&r2b_s);
                const double X[3] = {fma(hv, P[0], R[0]) - t->origin[0], fma(hv, P[1], R[1]) - t->origin[1],
                                     fma(hv, P[2], R[2]) - t->origin[2]};
                matvec_fma(t->M, X, b);
            } else {
                push_r(R, P, bc.s_cdt, bc.rs_cdt);
                trafo_transform_to(*fresh(&r2b_s), R, b);
            }
            R[0] = b[0];
            R[1] = b[1];
            R[2] = b[2];
            x[i] = R[0];
            y[i] = R[1];
            z[i] = R[2];
        }
        v[0] = fmin(v[0], R[0]);
        v[1] = fmin(v[1], R[1]);
        v[2] = fmin(v[2], R[2]);
        v[3] = fmin(v[3], -R[0]);
        v[4] = fmin(v[4], -R[1]);
        v[5] = fmin(v[5], -R[2]);
    }
    bounds_tail(bc, v, st, partials, ticket, g);
}

// Block minimum of the per-thread bounds v (min x, y, z, -max x, y, z) into
// partials[blk], then in the last block the bunch's bounds and its mesh
// (sharded: this rank's bounds for the exchange).
__device__ __forceinline__ void bounds_tail(const BunchConst& bc, double (&v)[6], StepState* st, double* partials,
                                            unsigned* ticket, VB g) {
    __shared__ double sm[6][kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = fmin(v[k], __shfl_down_sync(kFull, v[k], off));
    if (lane == 0)
        for (int k = 0; k < 6; ++k) sm[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        double m = INFINITY;
        for (int w = 0; w < kWarps; ++w) m = fmin(m, sm[threadIdx.x][w]);
        partials[(size_t)g.blk * 6 + threadIdx.x] = m;
    }
    if (!last_block(ticket, g.nblk)) return;
    __shared__ double tot[6];
    final_min<6>(partials, g.nblk, tot);
    __syncthreads();
    if (threadIdx.x == 0) {
        StepState& s = *st;
        if (bc.sharded) {  // this rank's bounds; k_finish_mesh completes after the exchange
            for (int k = 0; k < 6; ++k) s.bnd6[k] = tot[k];
        } else {
            for (int k = 0; k < 3; ++k) {
                s.bmin[k] = tot[k];
                s.bmax[k] = -tot[3 + k];
            }
            finish_mesh(s, bc);
        }
        *ticket = 0u;
    }
}
template <bool DRIFT, bool MIXED = false>
__global__ void __launch_bounds__(kThreads, 3) k_drift_to_beam(BunchConst bc, double* __restrict__ x, double* __restrict__ y,
                                                            double* __restrict__ z, const double* __restrict__ px,
                                                            const double* __restrict__ py, const double* __restrict__ pz,
                                                            StepState* st, double* partials, unsigned* ticket) {
    drift_body<DRIFT, MIXED>(bc, x, y, z, px, py, pz, st, partials, ticket, vb_grid());
}

// Streams this block's chunks (chunks blk, blk + nblk, ... of kStreamChunk
// elements) of NA double arrays through shared memory, double-buffered: the
// bulk copies of the next chunk are in flight while f(i, v) runs on every
// element i of the current one (v[a] = src[a][i], lane-contiguous reads).
// bar[0], bar[1] must be initialised barriers.  Returns false, with the
// copy-timeout flag raised, when a copy did not complete (every thread of the
// block returns false together, after waiting for its other copy).
constexpr int kStreamChunk = 512;

template <int NA>
__device__ __forceinline__ void stream_issue(const double* const (&src)[NA], long long N, long long c, double* buf,
                                             uint64_t* bar) {
    const long long first = c * kStreamChunk;
    const long long count = N - first < kStreamChunk ? N - first : kStreamChunk;
    double* dst[NA];
#pragma unroll
    for (int a = 0; a < NA; ++a) dst[a] = buf + a * kStreamChunk;
    stage_doubles<NA>(dst, src, first, count, bar);
}

template <int NA, typename F>
__device__ __forceinline__ bool stream_chunks(const double* const (&src)[NA], long long N, VB g, double* sm,
                                              uint64_t* bar, int* err, F&& f) {
    const long long nchunks = (N + kStreamChunk - 1) / kStreamChunk;
    if (g.blk < nchunks) stream_issue<NA>(src, N, g.blk, sm, &bar[0]);
    int k = 0;
    for (long long c = g.blk; c < nchunks; c += g.nblk, ++k) {
        const int b = k & 1;
        double* buf = sm + (size_t)b * NA * kStreamChunk;
        if (c + g.nblk < nchunks) stream_issue<NA>(src, N, c + g.nblk, sm + (size_t)(b ^ 1) * NA * kStreamChunk,
                                                   &bar[b ^ 1]);
        if (__syncthreads_or(!mbar_wait(&bar[b], (unsigned)(k >> 1) & 1u))) {
            if (threadIdx.x == 0) atomicOr(err, kFlagCopy);
            if (c + g.nblk < nchunks) mbar_wait(&bar[b ^ 1], (unsigned)((k + 1) >> 1) & 1u);
            return false;
        }
        const long long first = c * kStreamChunk;
        const int count = (int)(N - first < kStreamChunk ? N - first : kStreamChunk);
        const int body = count & ~1;
        for (int j = threadIdx.x; j < count; j += blockDim.x) {
            double v[NA];
            if (j < body) {
#pragma unroll
                for (int a = 0; a < NA; ++a) v[a] = buf[a * kStreamChunk + j];
            } else {
#pragma unroll
                for (int a = 0; a < NA; ++a) v[a] = src[a][first + j];
            }
            f(first + j, v);
        }
        __syncthreads();  // buffer b is read before the copies two chunks on land in it
    }
    return true;
}

// The reference particle needs no particle data: it runs beside the deposit.
__device__ __forceinline__ void advance_reference_body(const BunchConst& bc, StepState* st, VB g) {
    if (threadIdx.x == 0 && g.blk == 0)
        if (!advance_reference(*st, bc)) atomicOr(&st->err, kFlagFrame);
}
__global__ void k_advance_reference(BunchConst bc, StepState* st) { advance_reference_body(bc, st, vb_grid()); }

// ------------------------------------------------------------ cell keys
// key = lgp_x + n0 * (lgp_y + n1 * lgp_z) and the particle's rank among the
// particles of its cell (the first pass of the counting sort).
__global__ void __launch_bounds__(kThreads) k_cell_keys(BunchConst bc, const double* __restrict__ x,
                                                        const double* __restrict__ y, const double* __restrict__ z,
                                                        StepState* st, uint32_t* __restrict__ keys,
                                                        uint32_t* __restrict__ ranks, int* __restrict__ count) {
    __shared__ MeshConsts ms;
    load_mesh_consts(ms, st);
    __syncthreads();
    bool bad = false;
    const int lane = threadIdx.x & 31;
    // warp-uniform trip count: every lane takes part in the match below
    for (long long i0 = (long long)blockIdx.x * blockDim.x; i0 < bc.N; i0 += (long long)gridDim.x * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        const bool valid = i < bc.N;
        uint32_t key = 0xffffffffu;
        if (valid) {
            double X[3] = {x[i], y[i], z[i]};
            int l[3];
            double d[3];
            const MeshConsts* m = fresh(&ms);
            if (!cic_locate_r(m->hr, m->rhr, m->org, bc.n, X, l, d, bc.pz)) bad = true;
            const int lz = l[2] < 0 ? 0 : l[2];  // a DC beam's guard plane -1 sorts with plane 0
            key = (uint32_t)l[0] + (uint32_t)bc.n[0] * ((uint32_t)l[1] + (uint32_t)bc.n[1] * (uint32_t)lz);
            keys[i] = key;
        }
        // one atomic per distinct key in the warp; lanes take consecutive ranks
        const unsigned peers = __match_any_sync(kFull, key);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (valid && lane == leader) base = atomicAdd(&count[key], __popc(peers));
        base = __shfl_sync(kFull, base, leader);
        if (valid) ranks[i] = (uint32_t)(base + __popc(peers & ((1u << lane) - 1u)));
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
}

// ------------------------------------------------------------ deposit
// CIC cell and offset in units of the spacing: u = (x - origin) / h, cell
// centres at u = l + 1/2; false when the stencil would leave the mesh.
__device__ __forceinline__ bool cic_locate_fast(const double* rhr, const double* org, const int* n, const double* x,
                                                int* l, float* d, int pz) {
    bool ok = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const double u = fma(x[a] - org[a], rhr[a], -0.5);
        const double f = floor(u);
        int li = (int)f;
        float di = (float)(u - f);
        const int g = a == 2 ? pz : 0;  // a DC beam's z guard planes
        if (li < -g) {
            ok = false;
            li = -g;
        }
        if (li > n[a] - 2 + g) {
            ok = false;
            li = n[a] - 2 + g;
        }
        l[a] = li;
        d[a] = di;
    }
    return ok;
}
// CIC weights of one particle for the 8 corners, in IntCIC.h:850-857 order:
// (0,0,0) (1,0,0) (0,1,0) (1,1,0) (0,0,1) (1,0,1) (0,1,1) (1,1,1).
__device__ __forceinline__ void cic_charge(const double* d, double q, double* v) {
    v[0] = (1 - d[0]) * (1 - d[1]) * (1 - d[2]) * q;
    v[1] = d[0] * (1 - d[1]) * (1 - d[2]) * q;
    v[2] = (1 - d[0]) * d[1] * (1 - d[2]) * q;
    v[3] = d[0] * d[1] * (1 - d[2]) * q;
    v[4] = (1 - d[0]) * (1 - d[1]) * d[2] * q;
    v[5] = d[0] * (1 - d[1]) * d[2] * q;
    v[6] = (1 - d[0]) * d[1] * d[2] * q;
    v[7] = d[0] * d[1] * d[2] * q;
}

// Exact sums of the scattered charges (kFxFrac, fx_exponent, node_density in
// sc_exact.cuh).

// A fixed-point charge t = rint(v) (|t| < 2^51; the conversion rounds half
// to even, as rint) as two exact 32-bit limbs: hi = floor(t / 2^26) in
// [-2^25, 2^25) (arithmetic shift), lo = t - hi 2^26 in [0, 2^26).  Sums of
// up to 32 limbs fit 32 bits (|sum hi| < 2^30, sum lo < 2^31) and recombine
// exactly in 64 bits.
struct Limbs {
    int hi;
    unsigned lo;
};
__device__ __forceinline__ Limbs limbs_of(double v) {
    const long long t = __double2ll_rn(v);
    return Limbs{(int)(t >> 26), (unsigned)(t & 0x3ffffffll)};
}
__device__ __forceinline__ long long join(long long hi, long long lo) { return hi * (1ll << 26) + lo; }

// Group passes per warp before a warp falls back to per-lane additions.
constexpr int kMaxGroupPasses = 4;

// Node accumulator: two 64-bit words (L, H) holding the value H 2^32 + L.
// A group sum v (|v| < 2^57: up to 64 charges below 2^51) adds its low 32
// bits to L and its arithmetic high part v >> 32 to H, both as
// fire-and-forget atomics (no returned value is waited for).  L stays below
// 2^64 for fewer than 2^32 additions; H is a signed sum of terms below 2^25.  Integer additions commute, so the value
// is the same in any order.
__device__ __forceinline__ void acc_add(unsigned long long* a, long long v) {
    atomicAdd(a, (unsigned long long)v & 0xffffffffull);
    atomicAdd(a + 1, (unsigned long long)(v >> 32));
}

// Charge deposit.  Each warp takes 32 consecutive particles (the arrays are
// kept in cell order, so they share few cells), locates them (IntCIC.h:818-858),
// groups the lanes by cell (match.any) and sums each of the 8 corner charges
// over the group exactly (fixed point, full-warp redux.sync, one pass per
// group of two or more lanes).  The group's first lane adds the 8 sums to the
// node accumulators.  A sorted warp spans 2-3 cells on average at 1M
// particles / 64^3; warps with more than kMaxGroupPasses multi-lane groups
// (sparse regions) add per lane.  No floating-point value is accumulated by
// an atomic.
//
// With energy bins (BINNED) the key is bin * n^3 + cell: every active bin's
// charge goes to its own accumulators in the same pass, particles of bins
// not yet emitted deposit nothing (setBinCharge, PartBunchBase.hpp:722-725).
//
// A DC beam (PZ) first takes each particle through the periodic boundary
// along z (boundp's update(), the first use of the step's mesh; a wrapped
// position is written back) and drops the corner charges that land in the z
// guard planes -1 and n: the reference's single-rank scatter writes them
// into the guard layer, which ParticleAttrib::scatter zeroed and
// accumGuardCells (BareField.hpp:1013-1079) carries only into neighbouring
// local fields, of which one vnode has none (ParticleAttrib.h:207-221).
template <bool BINNED, bool PZ = false>
__device__ __forceinline__ void deposit_body(const BunchConst& bc, const double* __restrict__ x,
                                             const double* __restrict__ y, double* __restrict__ z,
                                             const int* __restrict__ bin, int nactive, StepState* st,
                                             unsigned long long* __restrict__ acc, VB g) {
    __shared__ MeshConsts ms;
    __shared__ double qdt_s, to_int_s;
    load_mesh_consts(ms, st);
    if (threadIdx.x == 0) {
        qdt_s = st->qdt;
        to_int_s = ldexp(1.0, kFxFrac - fx_exponent(st->qdt));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int nx = bc.n[0], nxy = bc.n[0] * bc.n[1];
    const uint32_t M = (uint32_t)nxy * (uint32_t)bc.n[2];
    bool bad = false;
    for (long long i0 = (long long)g.blk * blockDim.x; i0 < bc.N; i0 += (long long)g.nblk * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        int bk = 0;
        if constexpr (BINNED) bk = i < bc.N ? bin[i] : -1;
        const bool valid = i < bc.N && (!BINNED || (unsigned)bk < (unsigned)nactive);
        uint32_t key = 0xffffffffu;
        int lz = 0;  // z of the lower corner plane (DC beam: -1 .. n-1)
        double c[8];
        if (valid) {
            double X[3] = {x[i], y[i], z[i]};
            int l[3];
            double d[3];
            const MeshConsts* m = fresh(&ms);
            if constexpr (PZ) {
                const double w = wrap_z(X[2], m->org[2], m->org[2] + m->hr[2] * (double)bc.n[2]);
                if (w != X[2]) {
                    z[i] = w;
                    X[2] = w;
                }
            }
            if (!cic_locate_r(m->hr, m->rhr, m->org, bc.n, X, l, d, PZ ? 1 : 0)) bad = true;
            cic_charge(d, *fresh(&qdt_s), c);
            key = (uint32_t)(l[0] + nx * l[1] + nxy * l[2]) + (uint32_t)bk * M;
            lz = l[2];
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) c[k] = 0.0;
        }
        const double to_int = *fresh(&to_int_s);
        Limbs t[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) t[k] = limbs_of(c[k] * to_int);
        const unsigned group = __match_any_sync(kFull, key);
        const int gsize = __popc(group);
        const bool leader = lane == __ffs(group) - 1;
        // Groups of two or more lanes are summed one group per pass with
        // full-warp redux.sync (lanes outside the group add zero); a redux
        // whose mask differs between lanes would run once per distinct mask.
        unsigned multi = __ballot_sync(kFull, leader && gsize > 1);
        const bool passes = __popc(multi) <= kMaxGroupPasses;
        // single lanes, and every lane of a warp with many small groups,
        // add their own charges
        if (valid && (gsize == 1 || !passes)) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int node = (int)key + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                if (!PZ || (unsigned)(lz + (k >> 2)) < (unsigned)bc.n[2])
                    acc_add(acc + 2 * (long long)node, join(t[k].hi, t[k].lo));
            }
        }
        while (passes && multi) {
            const int ld = __ffs(multi) - 1;
            multi &= multi - 1;
            const bool in = (__shfl_sync(kFull, group, ld) >> lane) & 1u;
            long long s[8];
#pragma unroll
            for (int k = 0; k < 8; ++k)
                s[k] = join(__reduce_add_sync(kFull, in ? t[k].hi : 0), __reduce_add_sync(kFull, in ? t[k].lo : 0u));
            if (valid && lane == ld) {
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int node = (int)key + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                    if (!PZ || (unsigned)(lz + (k >> 2)) < (unsigned)bc.n[2]) acc_add(acc + 2 * (long long)node, s[k]);
                }
            }
        }
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
}
// The charge deposit of a bunch without bins or periodic z, two particles per
// lane: a warp takes 64 consecutive (cell-ordered) particles, lane l the
// pair 2l, 2l + 1 (one 16-byte load per coordinate).  A pair in one cell
// enters the warp's group reduction as the sum of its two fixed-point
// charges (|t_a + t_b| < 2^52, split into a 27-bit low limb and the signed
// rest, so 32 lanes' limb sums fit 32 bits), which halves the reduction
// passes per particle where cells are dense; the second particle of a pair
// that straddles a cell boundary adds its own charges.  The node values are
// the same integer sums as deposit_body's, so rho has the same bits.
__device__ __forceinline__ void deposit_pairs_body(const BunchConst& bc, const double* __restrict__ x,
                                                   const double* __restrict__ y, const double* __restrict__ z,
                                                   StepState* st, unsigned long long* __restrict__ acc, VB g) {
    __shared__ MeshConsts ms;
    __shared__ double qdt_s, to_int_s;
    load_mesh_consts(ms, st);
    if (threadIdx.x == 0) {
        qdt_s = st->qdt;
        to_int_s = ldexp(1.0, kFxFrac - fx_exponent(st->qdt));
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nx = bc.n[0], nxy = bc.n[0] * bc.n[1];
    const long long span = 2ll * blockDim.x;
    bool bad = false;
    for (long long i0 = (long long)g.blk * span; i0 < bc.N; i0 += (long long)g.nblk * span) {
        const long long ia = i0 + 64ll * warp + 2 * lane, ib = ia + 1;
        const bool va = ia < bc.N, vb = ib < bc.N;
        double Xa[3] = {0.0, 0.0, 0.0}, Xb[3] = {0.0, 0.0, 0.0};
        if (vb) {  // ia is even: the pair is one aligned 16-byte load per coordinate
            const double2 px = *reinterpret_cast<const double2*>(x + ia);
            const double2 py = *reinterpret_cast<const double2*>(y + ia);
            const double2 pz = *reinterpret_cast<const double2*>(z + ia);
            Xa[0] = px.x, Xa[1] = py.x, Xa[2] = pz.x;
            Xb[0] = px.y, Xb[1] = py.y, Xb[2] = pz.y;
        } else if (va) {
            Xa[0] = x[ia], Xa[1] = y[ia], Xa[2] = z[ia];
        }
        uint32_t ka = 0xffffffffu, kb = 0xfffffffeu;
        int la[3], lb[3];
        double da[3], db[3];
        const MeshConsts* m = fresh(&ms);
        if (va) {
            if (!cic_locate_r(m->hr, m->rhr, m->org, bc.n, Xa, la, da)) bad = true;
            ka = (uint32_t)(la[0] + nx * la[1] + nxy * la[2]);
        }
        if (vb) {
            if (!cic_locate_r(m->hr, m->rhr, m->org, bc.n, Xb, lb, db)) bad = true;
            kb = (uint32_t)(lb[0] + nx * lb[1] + nxy * lb[2]);
        }
        const bool same = vb && ka == kb;
        const double q = *fresh(&qdt_s), to_int = *fresh(&to_int_s);
        long long T[8];
        {
            double c[8];
            if (va) {
                cic_charge(da, q, c);
            } else {
#pragma unroll
                for (int k = 0; k < 8; ++k) c[k] = 0.0;
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) T[k] = __double2ll_rn(c[k] * to_int);
        }
        if (vb) {
            double c[8];
            cic_charge(db, q, c);
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const long long t = __double2ll_rn(c[k] * to_int);
                if (same) {
                    T[k] += t;
                } else {
                    const int node = (int)kb + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                    acc_add(acc + 2 * (long long)node, t);
                }
            }
        }
        const unsigned group = __match_any_sync(kFull, ka);
        const int gsize = __popc(group);
        const bool leader = lane == __ffs(group) - 1;
        unsigned multi = __ballot_sync(kFull, leader && gsize > 1);
        const bool passes = __popc(multi) <= kMaxGroupPasses;
        if (va && (gsize == 1 || !passes)) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int node = (int)ka + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                acc_add(acc + 2 * (long long)node, T[k]);
            }
        }
        while (passes && multi) {
            const int ld = __ffs(multi) - 1;
            multi &= multi - 1;
            const bool in = (__shfl_sync(kFull, group, ld) >> lane) & 1u;
            long long sum[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int hi = __reduce_add_sync(kFull, in ? (int)(T[k] >> 27) : 0);
                const unsigned lo = __reduce_add_sync(kFull, in ? (unsigned)(T[k] & 0x7ffffffll) : 0u);
                sum[k] = (long long)hi * (1ll << 27) + (long long)lo;
            }
            if (va && lane == ld) {
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int node = (int)ka + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                    acc_add(acc + 2 * (long long)node, sum[k]);
                }
            }
        }
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
}

template <bool PZ>
__global__ void __launch_bounds__(kThreads) k_deposit(BunchConst bc, const double* __restrict__ x, const double* __restrict__ y,
                                                      double* __restrict__ z, StepState* st,
                                                      unsigned long long* __restrict__ acc) {
    if constexpr (PZ)
        deposit_body<false, true>(bc, x, y, z, nullptr, 0, st, acc, vb_grid());
    else
        deposit_pairs_body(bc, x, y, z, st, acc, vb_grid());
}
__global__ void __launch_bounds__(kThreads) k_deposit_bins(BunchConst bc, const double* __restrict__ x,
                                                           const double* __restrict__ y, double* __restrict__ z,
                                                           const int* __restrict__ bin, int nactive, StepState* st,
                                                           unsigned long long* __restrict__ acc) {
    deposit_body<true>(bc, x, y, z, bin, nactive, st, acc, vb_grid());
}

// The mixed form's deposit.  The cell and offset come from the FP64 position
// (cic_locate_fast, as in the mixed gather), the eight CIC weights are FP32
// products, and each weight w <= 1 becomes the integer rint(w 2^26): the sum
// over a lane group of up to 32 fits one 32-bit word, so a group pass is one
// full-warp redux.sync per corner (half the passes of the two charge limbs)
// and the group's first lane adds one 64-bit atomic per corner to the low
// word of the node accumulator (the high word stays zero).  A node then holds
// the exact, order-independent sum of its quantised weights; the assembly
// multiplies it by Q dt 2^-26.  The DC beam's z boundary and guard planes as
// in deposit_body.
constexpr int kWeightFrac = 26;

template <bool PZ>
__device__ __forceinline__ void deposit_mixed_body(const BunchConst& bc, const double* __restrict__ x,
                                                   const double* __restrict__ y, double* __restrict__ z, StepState* st,
                                                   unsigned long long* __restrict__ acc, VB g) {
    __shared__ MeshConsts ms;
    load_mesh_consts(ms, st);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int nx = bc.n[0], nxy = bc.n[0] * bc.n[1];
    const float scale = 0x1p26f;
    bool bad = false;
    for (long long i0 = (long long)g.blk * blockDim.x; i0 < bc.N; i0 += (long long)g.nblk * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        const bool valid = i < bc.N;
        uint32_t key = 0xffffffffu;
        int lz = 0;
        unsigned t[8];
        if (valid) {
            double X[3] = {x[i], y[i], z[i]};
            const MeshConsts* m = fresh(&ms);
            if constexpr (PZ) {
                const double w = wrap_z(X[2], m->org[2], m->org[2] + m->hr[2] * (double)bc.n[2]);
                if (w != X[2]) {
                    z[i] = w;
                    X[2] = w;
                }
            }
            int l[3];
            float d[3];
            if (!cic_locate_fast(m->rhr, m->org, bc.n, X, l, d, PZ ? 1 : 0)) bad = true;
            const float u[3] = {1.0f - d[0], 1.0f - d[1], 1.0f - d[2]};
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const float w = (k & 1 ? d[0] : u[0]) * (k & 2 ? d[1] : u[1]) * (k & 4 ? d[2] : u[2]);
                t[k] = __float2uint_rn(w * scale);
            }
            key = (uint32_t)(l[0] + nx * l[1] + nxy * l[2]);
            lz = l[2];
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) t[k] = 0u;
        }
        const unsigned group = __match_any_sync(kFull, key);
        const int gsize = __popc(group);
        const bool leader = lane == __ffs(group) - 1;
        unsigned multi = __ballot_sync(kFull, leader && gsize > 1);
        const bool passes = __popc(multi) <= kMaxGroupPasses;
        if (valid && (gsize == 1 || !passes)) {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int node = (int)key + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                if ((!PZ || (unsigned)(lz + (k >> 2)) < (unsigned)bc.n[2]) && t[k])
                    atomicAdd(acc + 2 * (long long)node, (unsigned long long)t[k]);
            }
        }
        while (passes && multi) {
            const int ld = __ffs(multi) - 1;
            multi &= multi - 1;
            const bool in = (__shfl_sync(kFull, group, ld) >> lane) & 1u;
            unsigned sum[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) sum[k] = __reduce_add_sync(kFull, in ? t[k] : 0u);
            if (valid && lane == ld) {
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int node = (int)key + (k & 1) + ((k >> 1) & 1) * nx + ((k >> 2) & 1) * nxy;
                    if ((!PZ || (unsigned)(lz + (k >> 2)) < (unsigned)bc.n[2]) && sum[k])
                        atomicAdd(acc + 2 * (long long)node, (unsigned long long)sum[k]);
                }
            }
        }
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
}
template <bool PZ>
__global__ void __launch_bounds__(kThreads) k_deposit_mixed(BunchConst bc, const double* __restrict__ x,
                                                            const double* __restrict__ y, double* __restrict__ z,
                                                            StepState* st, unsigned long long* __restrict__ acc) {
    deposit_mixed_body<PZ>(bc, x, y, z, st, acc, vb_grid());
}

// rho = (exact node sum) / dT * tmp2   (PartBunch.cpp:496, :510-511); the
// accumulators are cleared for the next deposit.  `weights`: the node values
// are sums of 26-bit CIC weights (the mixed deposit), in units of Q dt 2^-26.
template <typename T>
__device__ __forceinline__ void assemble_body(const BunchConst& bc, const StepState* __restrict__ st,
                                              unsigned long long* __restrict__ acc, T* __restrict__ rho, VB g,
                                              bool weights) {
    const int M = bc.n[0] * bc.n[1] * bc.n[2];
    const double dT = bc.dT, tmp2 = st->tmp2;
    const double unit = weights ? ldexp(st->qdt, -kWeightFrac) : ldexp(1.0, fx_exponent(st->qdt) - kFxFrac);
    for (int c = g.blk * blockDim.x + threadIdx.x; c < M; c += g.nblk * blockDim.x) {
        const double s = node_density(reinterpret_cast<const ulonglong2*>(acc)[c], unit, dT, tmp2);
        rho[c] = (T)s;
        reinterpret_cast<ulonglong2*>(acc)[c] = make_ulonglong2(0ull, 0ull);
    }
}
template <typename T>
__global__ void __launch_bounds__(kThreads) k_assemble_rho(BunchConst bc, const StepState* __restrict__ st,
                                                           unsigned long long* __restrict__ acc, T* __restrict__ rho,
                                                           int weights) {
    assemble_body<T>(bc, st, acc, rho, vb_grid(), weights != 0);
}

// ------------------------------------------------------------ Green's function
// The antiderivative of (FFTPoissonSolver.cpp:472-493) in the reference's
// operation order, with atan and log evaluated in double-double and rounded
// once (sc_ddmath.cuh): correctly rounded except in rare near-tie cases, so
// G does not carry the device library's last-bit differences into the
// eight-corner cancellation.
// CR: the correctly rounded double-double atan / log of the plain form;
// otherwise CUDA's own FP64 atan / log (a few ulp), the mixed form's
// Green's function, still FP64 throughout.
template <bool CR = true>
__device__ __forceinline__ double igf_antiderivative(double x, double y, double z, double cellVolume) {
    double r = sqrt(x * x + y * y + z * z);
    if constexpr (CR) {
        double tmpgrn = -z * z * ddm::atan_dd(x * y / (z * r)) / 2;
        tmpgrn += -y * y * ddm::atan_dd(x * z / (y * r)) / 2;
        tmpgrn += -x * x * ddm::atan_dd(y * z / (x * r)) / 2;
        tmpgrn += y * z * ddm::log_dd(x + r);
        tmpgrn += x * z * ddm::log_dd(y + r);
        tmpgrn += x * y * ddm::log_dd(z + r);
        return tmpgrn / cellVolume;
    } else {
        double tmpgrn = -z * z * atan(x * y / (z * r)) / 2;
        tmpgrn += -y * y * atan(x * z / (y * r)) / 2;
        tmpgrn += -x * x * atan(y * z / (x * r)) / 2;
        tmpgrn += y * z * log(x + r);
        tmpgrn += x * z * log(y + r);
        tmpgrn += x * y * log(z + r);
        return tmpgrn / cellVolume;
    }
}

template <bool CR = true>
__device__ __forceinline__ void igf_tmp_body(int n0, int n1, int n2, const StepState* __restrict__ st,
                                             double* __restrict__ tmp, VB g) {
    const int t0 = n0 + 2, t1 = n1 + 2, t2 = n2 + 2;
    const double h0 = st->hr_scaled[0], h1 = st->hr_scaled[1], h2 = st->hr_scaled[2];
    const double cellVolume = h0 * h1 * h2;
    for (int c = g.blk * blockDim.x + threadIdx.x; c < t0 * t1 * t2; c += g.nblk * blockDim.x) {
        const int i = c % t0, j = (c / t0) % t1, k = c / (t0 * t1);
        const double vx = i * h0 - h0 / 2;
        const double vy = j * h1 - h1 / 2;
        const double vz = k * h2 - h2 / 2;
        tmp[c] = igf_antiderivative<CR>(vx, vy, vz, cellVolume);
    }
}
template <bool CR = true>
__global__ void __launch_bounds__(kThreads) k_igf_tmp(int n0, int n1, int n2, const StepState* __restrict__ st,
                                                      double* __restrict__ tmp) {
    igf_tmp_body<CR>(n0, n1, n2, st, tmp, vb_grid());
}

// G on (n0+1)(n1+1)(n2+1) points, 8-corner difference (:508-516), then
// G[0,0,0] <- G[0,0,1] (mirrorRhoField, :657).
__device__ __forceinline__ void igf_G_body(int n0, int n1, int n2, const double* __restrict__ tmp,
                                           double* __restrict__ G, VB g) {
    const int g0 = n0 + 1, g1 = n1 + 1, g2 = n2 + 1;
    const int t0 = n0 + 2, t1 = n1 + 2;
    for (int c = g.blk * blockDim.x + threadIdx.x; c < g0 * g1 * g2; c += g.nblk * blockDim.x) {
        const int i = c % g0, j = (c / g0) % g1, k = c / (g0 * g1);
        G[c] = igf_G_at(tmp, t0, t1, i, j, k);
    }
}
__global__ void __launch_bounds__(kThreads) k_igf_G(int n0, int n1, int n2, const double* __restrict__ tmp,
                                                    double* __restrict__ G) {
    igf_G_body(n0, n1, n2, tmp, G, vb_grid());
}

// ------------------------------------------------------------ sharded bunch
// Tails of the reductions once the ranks' partial results have been combined
// (bounds by min, exact sums as integer limbs), on one thread.
__global__ void k_finish_mesh(BunchConst bc, StepState* st) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    StepState& s = *st;
    for (int k = 0; k < 3; ++k) {
        s.bmin[k] = s.bnd6[k];
        s.bmax[k] = -s.bnd6[3 + k];
    }
    finish_mesh(s, bc);
}

// psum from the combined limbs; frame: the beam frame of the next step
// (derive_beam_frame); advance: the step counter of the gather.
__global__ void k_finish_psum(BunchConst bc, StepState* st, int frame, int advance) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    StepState& s = *st;
    for (int k = 0; k < 3; ++k) s.psum[k] = ex_to_double(get_limbs(s.xlimbs + 4 * k));
    if (frame && !derive_beam_frame(s, bc)) atomicOr(&s.err, kFlagFrame);
    if (advance) s.step += 1;
}

__global__ void k_finish_stats(StepState* st) {
    if (blockIdx.x != 0 || threadIdx.x >= 28) return;
    const double v = ex_to_double(get_limbs(st->xlimbs + 4 * threadIdx.x));
    if (threadIdx.x < 27)
        st->moments[threadIdx.x] = v;
    else
        st->gsum = v;
}

// ------------------------------------------------------------ image charge
// Antiderivative planes of the image's Green's function
// (shiftedIntGreensFunction, FFTPoissonSolver.cpp:556-596): set 0 at
// z = k hz - hz/2 + zshift (tmpgreen), set 1 at z = k hz - hz/2 + zshift - n2 hz
// (grn2), k in [0, n2+1]; x, y as in the unshifted function.  hz and zshift
// are the bin's (st->hr_scaled, st->zshift).
__global__ void __launch_bounds__(kThreads) k_igf_tmp_img(int n0, int n1, int n2, const StepState* __restrict__ st,
                                                          double* __restrict__ tmp) {
    const int t0 = n0 + 2, t1 = n1 + 2, t2 = n2 + 2;
    const int T3 = t0 * t1 * t2;
    const double h0 = st->hr_scaled[0], h1 = st->hr_scaled[1], h2 = st->hr_scaled[2];
    const double zshift = st->zshift;
    const double cellVolume = h0 * h1 * h2;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < 2 * T3; c += gridDim.x * blockDim.x) {
        const int set = c >= T3 ? 1 : 0;
        const int r = c - set * T3;
        const int i = r % t0, j = (r / t0) % t1, k = r / (t0 * t1);
        const double vx = i * h0 - h0 / 2;
        const double vy = j * h1 - h1 / 2;
        double vz = k * h2 - h2 / 2 + zshift;
        if (set) vz = vz - n2 * h2;
        tmp[c] = igf_antiderivative(vx, vy, vz, cellVolume);
    }
}

// The image's G on (n0+1)(n1+1)(2 n2), x fastest: z index k <= n2 is the
// eight-corner sum of set 0 at k (rho2[I][J][K], :598-607), k > n2 that of
// set 1 at k - n2 (mirrorRhoField(ggrn2), :672-676).  Mirrored in x and y
// only, so the cosine transforms cover x, y and z takes a full real
// transform.  No G[0,0,0] overwrite.
__global__ void __launch_bounds__(kThreads) k_igf_G_img(int n0, int n1, int n2, const double* __restrict__ tmp,
                                                        double* __restrict__ G) {
    const int g0 = n0 + 1, g1 = n1 + 1, L2 = 2 * n2;
    const int t0 = n0 + 2, t1 = n1 + 2;
    const int T3 = t0 * t1 * (n2 + 2);
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < g0 * g1 * L2; c += gridDim.x * blockDim.x) {
        const int i = c % g0, j = (c / g0) % g1, kk = c / (g0 * g1);
        const double* t = kk <= n2 ? tmp : tmp + T3;
        const int k = kk <= n2 ? kk : kk - n2;
#define TG(a, b, e) t[(a) + t0 * ((b) + t1 * (e))]
        double g = TG(i + 1, j + 1, k + 1);
        g += TG(i + 1, j, k);
        g += TG(i, j + 1, k);
        g += TG(i, j, k + 1);
        g -= TG(i + 1, j + 1, k);
        g -= TG(i + 1, j, k + 1);
        g -= TG(i, j + 1, k + 1);
        g -= TG(i, j, k);
#undef TG
        G[c] = g;
    }
}

// ------------------------------------------------------------ energy bins
// calcGammas (PartBunchBase.hpp:639-683): per bin the sum of sqrt(1 + P.P)
// and the particle count.  The sum is exact: gamma as the 2^-72 fixed point
// of sc_exact.cuh (below 2^96 for gamma < 2^24) in six 16-bit limbs.  Lanes
// of a warp with the same bin (match.any) sum their limbs with redux.sync
// (at most 32 * 2^16 < 2^21 per limb) and the group's first lane adds them
// to its warp's 64-bit shared counters, so no carry is lost for fewer than
// 2^48 particles and the mean does not depend on the particle order.  The
// last block sums the block partials (one column per thread) and
// writes each bin's StepState: this step's mesh with the bin's gamma and the
// scalars of computeSelfFields(bin) (PartBunch.cpp:173-185, :246-249).
constexpr int kGammaLimbs = 6;
constexpr int kGammaCols = kGammaLimbs + 1;  // limbs and the count
__global__ void __launch_bounds__(kThreads) k_bin_gammas(BunchConst bc, const double* __restrict__ px,
                                                         const double* __restrict__ py, const double* __restrict__ pz,
                                                         const int* __restrict__ bin, int nbins, StepState* st,
                                                         StepState* __restrict__ bst,
                                                         unsigned long long* __restrict__ partials, unsigned* ticket) {
    // one set of counters per warp: a warp's group leaders hold distinct
    // bins, so they add without atomics
    __shared__ unsigned long long acc[kWarps][kMaxBins * kGammaCols];
    const int ncol = nbins * kGammaCols;
    for (int e = threadIdx.x; e < kWarps * kMaxBins * kGammaCols; e += blockDim.x) (&acc[0][0])[e] = 0ull;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    bool bad = false;
    for (long long i0 = blockIdx.x * (long long)blockDim.x; i0 < bc.N; i0 += (long long)gridDim.x * blockDim.x) {
        const long long i = i0 + threadIdx.x;
        int b = -1;
        unsigned limb[kGammaLimbs] = {0u, 0u, 0u, 0u, 0u, 0u};
        if (i < bc.N) {
            b = bin[i];
            if ((unsigned)b >= (unsigned)nbins) {
                bad = true;
                b = -1;
            } else {
                const double P[3] = {px[i], py[i], pz[i]};
                const u128 v = (u128)ex_from(sqrt(1.0 + dot3(P, P)));
#pragma unroll
                for (int q = 0; q < kGammaLimbs; ++q) limb[q] = (unsigned)(v >> (16 * q)) & 0xffffu;
            }
        }
        const unsigned group = __match_any_sync(kFull, b);
        unsigned sum[kGammaLimbs];
#pragma unroll
        for (int q = 0; q < kGammaLimbs; ++q) sum[q] = __reduce_add_sync(group, limb[q]);
        if (b >= 0 && lane == __ffs(group) - 1) {
            unsigned long long* a = acc[warp] + b * kGammaCols;
#pragma unroll
            for (int q = 0; q < kGammaLimbs; ++q) a[q] += (unsigned long long)sum[q];
            a[kGammaLimbs] += (unsigned long long)__popc(group);
        }
    }
    if (bad) atomicOr(&st->err, kFlagBin);
    __syncthreads();
    for (int e = threadIdx.x; e < ncol; e += blockDim.x) {
        unsigned long long t = 0ull;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) t += acc[w][e];
        partials[(size_t)blockIdx.x * ncol + e] = t;
    }
    if (!last_block(ticket, gridDim.x)) return;
    __shared__ unsigned long long tot[kMaxBins * kGammaCols];
    for (int e = threadIdx.x; e < ncol; e += blockDim.x) {
        unsigned long long t = 0ull;
        for (int k = 0; k < (int)gridDim.x; ++k) t += __ldcg(partials + (size_t)k * ncol + e);
        tot[e] = t;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
        const unsigned long long* t = tot + b * kGammaCols;
        u128 sum = 0;
#pragma unroll
        for (int q = 0; q < kGammaLimbs; ++q) sum += (u128)t[q] << (16 * q);
        const long long cnt = (long long)t[kGammaLimbs];
        double gz = ex_to_double((i128)sum);
        if (cnt != 0)
            gz /= (double)cnt;
        else
            gz = 1.0;
        // the fields the bin's kernels read (assemble, Green's functions,
        // pass E, gradient); the rest of the StepState is not used per bin
        StepState& o = bst[b];
        for (int d = 0; d < 3; ++d) {
            o.hr[d] = st->hr[d];
            o.rhr[d] = st->rhr[d];
            o.origin[d] = st->origin[d];
        }
        o.qdt = st->qdt;
        const double scaleFactor = 1;
        o.gammaz = gz;
        o.bin_count = cnt;
        o.tmp2 = 1 / st->hr[0] * 1 / st->hr[1] * 1 / st->hr[2] / (scaleFactor * scaleFactor * scaleFactor) / gz;
        o.hr_scaled[0] = st->hr[0] * scaleFactor;
        o.hr_scaled[1] = st->hr[1] * scaleFactor;
        o.hr_scaled[2] = st->hr[2] * scaleFactor;
        o.hr_scaled[2] *= gz;
        o.hvol = o.hr_scaled[0] * o.hr_scaled[1] * o.hr_scaled[2];
        o.betaC = sqrt(gz * gz - 1.0) / gz / kC;
        o.zshift = -(2 * st->origin[2] + (0 + (bc.n[2] - 1) + 1) * st->hr[2]) * gz * scaleFactor;
    }
    if (threadIdx.x == 0) *ticket = 0u;
}

// -grad phi (UniformCartesian.hpp:2129-2203, scaled by the bin's (g, g, 1/g),
// PartBunch.cpp:199-200) of one node of a potential.
__device__ __forceinline__ void neg_grad_scaled(const double* __restrict__ phi, int c, const int (&idx)[3],
                                                const int (&n)[3], const int (&stv)[3], const double (&id)[3],
                                                const double (&sc)[3], double (&e)[3]) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double* f = phi + c;
        const int s = stv[d];
        double g;
        if (idx[d] == 0)
            g = id[d] * (-1.0 * f[2 * s] + 4.0 * f[s] - 3.0 * f[0]);
        else if (idx[d] == n[d] - 1)
            g = id[d] * (1.0 * f[-2 * s] - 4.0 * f[-s] + 3.0 * f[0]);
        else
            g = id[d] * (f[s] - f[-s]);
        e[d] = (-g) * sc[d];
    }
}

// One bin's fields added into F8: first its own charge's E and B =
// (-betaC E_y, +betaC E_x) (:238-239), then its image's E and B = (+betaC
// E_y, -betaC E_x) (:426-427) -- the additions in the order of two separate
// passes, in one read and write of F8.
__global__ void __launch_bounds__(kThreads, 4) k_grad_acc(BunchConst bc, const StepState* __restrict__ st,
                                                       const double* __restrict__ phi,
                                                       const double* __restrict__ phi_img, double* __restrict__ F8) {
    const int n[3] = {bc.n[0], bc.n[1], bc.n[2]};
    const int M = n[0] * n[1] * n[2];
    const int stv[3] = {1, n[0], n[0] * n[1]};
    const double h[3] = {st->hr[0], st->hr[1], st->hr[2]};
    const double id[3] = {0.5 / h[0], 0.5 / h[1], 0.5 / h[2]};
    const double gz = st->gammaz;
    const double sc[3] = {gz / 1.0, gz / 1.0, 1.0 / (1.0 * gz)};
    const double betaC = st->betaC;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < M; c += gridDim.x * blockDim.x) {
        const int idx[3] = {c % n[0], (c / n[0]) % n[1], c / (n[0] * n[1])};
        double e[3], ei[3];
        neg_grad_scaled(phi, c, idx, n, stv, id, sc, e);
        neg_grad_scaled(phi_img, c, idx, n, stv, id, sc, ei);
        double* o = F8 + 8 * (size_t)c;
        double2 exy = *reinterpret_cast<const double2*>(o);
        double2 ez = *reinterpret_cast<const double2*>(o + 2);
        double2 bxy = *reinterpret_cast<const double2*>(o + 4);
        exy.x = exy.x + e[0];
        exy.y = exy.y + e[1];
        ez.x = ez.x + e[2];
        bxy.x = bxy.x - betaC * e[1];
        bxy.y = bxy.y + betaC * e[0];
        exy.x = exy.x + ei[0];
        exy.y = exy.y + ei[1];
        ez.x = ez.x + ei[2];
        bxy.x = bxy.x + betaC * ei[1];
        bxy.y = bxy.y - betaC * ei[0];
        *reinterpret_cast<double2*>(o) = exy;
        *reinterpret_cast<double2*>(o + 2) = ez;
        *reinterpret_cast<double2*>(o + 4) = bxy;
    }
}

// get_bounds of the particle positions (PartBunchBase.hpp:1178-1219) for the
// statistics: min of x, y, z and of -x, -y, -z into out[6] (exact, any order;
// the shards of a bunch combine by min).
__global__ void __launch_bounds__(kThreads) k_bounds(BunchConst bc, const double* __restrict__ x,
                                                     const double* __restrict__ y, const double* __restrict__ z,
                                                     double* partials, unsigned* ticket, double* __restrict__ out) {
    double v[6] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        const double R[3] = {x[i], y[i], z[i]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = fmin(v[d], R[d]);
            v[3 + d] = fmin(v[3 + d], -R[d]);
        }
    }
    __shared__ double sm[6][kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < 6; ++k) v[k] = fmin(v[k], __shfl_down_sync(kFull, v[k], off));
    if (lane == 0)
        for (int k = 0; k < 6; ++k) sm[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x < 6) {
        double m = INFINITY;
        for (int w = 0; w < kWarps; ++w) m = fmin(m, sm[threadIdx.x][w]);
        partials[(size_t)blockIdx.x * 6 + threadIdx.x] = m;
    }
    if (!last_block(ticket, gridDim.x)) return;
    __shared__ double tot[6];
    final_min<6>(partials, gridDim.x, tot);
    __syncthreads();
    if (threadIdx.x < 6) out[threadIdx.x] = tot[threadIdx.x];
    if (threadIdx.x == 0) *ticket = 0u;
}

// The state of the particle with original index `target` (R[0], P[0] of the statistics).
__global__ void __launch_bounds__(kThreads) k_find_id(const uint32_t* __restrict__ id, long long n, uint32_t target,
                                                      const double* __restrict__ x, const double* __restrict__ y,
                                                      const double* __restrict__ z, const double* __restrict__ px,
                                                      const double* __restrict__ py, const double* __restrict__ pz,
                                                      double* __restrict__ out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (id[i] == target) {
            out[0] = x[i];
            out[1] = y[i];
            out[2] = z[i];
            out[3] = px[i];
            out[4] = py[i];
            out[5] = pz[i];
        }
}

__global__ void __launch_bounds__(kThreads) k_bins_by_id(const int* __restrict__ host_order,
                                                         const uint32_t* __restrict__ id, int* __restrict__ bin,
                                                         long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        bin[i] = host_order[id[i]];
}

__global__ void __launch_bounds__(kThreads) k_permute_i32(const uint32_t* __restrict__ sval, const int* __restrict__ in,
                                                          int* __restrict__ out, long long n) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x)
        out[p] = in[sval[p]];
}

// ------------------------------------------------------------ gradient
// phi is FP64 in both forms; T is the storage type of the field.
template <typename T>
__device__ __forceinline__ void grad_body(const BunchConst& bc, const StepState* __restrict__ st,
                                          const double* __restrict__ phi, T* __restrict__ E4, VB g) {
    const int n[3] = {bc.n[0], bc.n[1], bc.n[2]};
    const int M = n[0] * n[1] * n[2];
    const int stv[3] = {1, n[0], n[0] * n[1]};
    const double h[3] = {st->hr[0], st->hr[1], st->hr[2]};
    const double id[3] = {0.5 / h[0], 0.5 / h[1], 0.5 / h[2]};
    const double gz = st->gammaz;
    const double sc[3] = {gz / 1.0, gz / 1.0, 1.0 / (1.0 * gz)};
    for (int c = g.blk * blockDim.x + threadIdx.x; c < M; c += g.nblk * blockDim.x) {
        const int idx[3] = {c % n[0], (c / n[0]) % n[1], c / (n[0] * n[1])};
        double e[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const double* f = phi + c;
            const int s = stv[d];
            double g;
            if (idx[d] == 0)
                g = id[d] * (-1.0 * (double)f[2 * s] + 4.0 * (double)f[s] - 3.0 * (double)f[0]);
            else if (idx[d] == n[d] - 1)
                g = id[d] * (1.0 * (double)f[-2 * s] - 4.0 * (double)f[-s] + 3.0 * (double)f[0]);
            else
                g = id[d] * ((double)f[s] - (double)f[-s]);
            e[d] = (-g) * sc[d];
        }
        E4[4 * (size_t)c + 0] = (T)e[0];
        E4[4 * (size_t)c + 1] = (T)e[1];
        E4[4 * (size_t)c + 2] = (T)e[2];
        E4[4 * (size_t)c + 3] = (T)0;
    }
}
template <typename T>
__global__ void __launch_bounds__(kThreads) k_grad(BunchConst bc, const StepState* __restrict__ st,
                                                   const double* __restrict__ phi, T* __restrict__ E4) {
    grad_body<T>(bc, st, phi, E4, vb_grid());
}

// ------------------------------------------------------------ gather, kick, push
// CIC gather (IntCIC.h:935-975): the eight weighted corner values added in
// the reference's order, accumulated as the corners are loaded.
// The corner planes along z: l and l + 1, or for a DC beam's guard planes
// their periodic images (PeriodicFace fills the guard layer before the
// gather, ParticleAttrib.h:297-299): plane -1 is plane n-1, plane n is 0.
__device__ __forceinline__ void corner_planes(const int* n, int lz, int (&zp)[2]) {
    zp[0] = lz < 0 ? n[2] - 1 : lz;
    zp[1] = lz + 1 >= n[2] ? 0 : lz + 1;
}

template <typename T>
__device__ __forceinline__ void cic_gather(const T* __restrict__ E4, const int* n, const int* l, const double* d,
                                           double* Ef) {
    const int nx = n[0], nxy = n[0] * n[1];
    int zp[2];
    corner_planes(n, l[2], zp);
    const int b = l[0] + nx * l[1];
    const double u[3] = {1 - d[0], 1 - d[1], 1 - d[2]};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int a0 = k & 1, a1 = (k >> 1) & 1, a2 = (k >> 2) & 1;
        const double w = (a0 ? d[0] : u[0]) * (a1 ? d[1] : u[1]) * (a2 ? d[2] : u[2]);
        const T* p = E4 + 4 * (size_t)(b + a0 + a1 * nx + zp[a2] * nxy);
        double e0, e1, e2;
        if constexpr (sizeof(T) == sizeof(double)) {
            const double2 a = *reinterpret_cast<const double2*>(p);  // nodes are 32-byte aligned
            e0 = a.x;
            e1 = a.y;
            e2 = (double)p[2];
        } else {
            const float4 a = *reinterpret_cast<const float4*>(p);  // nodes are 16-byte aligned
            e0 = (double)a.x;
            e1 = (double)a.y;
            e2 = (double)a.z;
        }
        if (k == 0) {
            Ef[0] = w * e0;
            Ef[1] = w * e1;
            Ef[2] = w * e2;
        } else {
            Ef[0] = Ef[0] + w * e0;
            Ef[1] = Ef[1] + w * e1;
            Ef[2] = Ef[2] + w * e2;
        }
    }
}

// The energy-bin form gathers E and B from the summed field of all bins and
// images, F8 = (Ex, Ey, Ez, -, Bx, By, -, -) per node (64-byte aligned).
// Ef += Eftmp and Bf +-= betaC Eftmp of every bin (PartBunch.cpp:238-244,
// :417-427) are linear in the gathered values, so summing the nodes first
// gives the same fields up to the order of the additions.
__device__ __forceinline__ void cic_gather8(const double* __restrict__ F8, const int* n, const int* l, const double* d,
                                            double* Eb, double* Bb) {
    const int nx = n[0], nxy = n[0] * n[1];
    const int b = l[0] + nx * l[1] + nxy * l[2];
    const double u[3] = {1 - d[0], 1 - d[1], 1 - d[2]};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int a0 = k & 1, a1 = (k >> 1) & 1, a2 = (k >> 2) & 1;
        const double w = (a0 ? d[0] : u[0]) * (a1 ? d[1] : u[1]) * (a2 ? d[2] : u[2]);
        const double* p = F8 + 8 * (size_t)(b + a0 + a1 * nx + a2 * nxy);
        const double2 exy = *reinterpret_cast<const double2*>(p);
        const double ez = p[2];
        const double2 bxy = *reinterpret_cast<const double2*>(p + 4);
        if (k == 0) {
            Eb[0] = w * exy.x;
            Eb[1] = w * exy.y;
            Eb[2] = w * ez;
            Bb[0] = w * bxy.x;
            Bb[1] = w * bxy.y;
        } else {
            Eb[0] = Eb[0] + w * exy.x;
            Eb[1] = Eb[1] + w * exy.y;
            Eb[2] = Eb[2] + w * ez;
            Bb[0] = Bb[0] + w * bxy.x;
            Bb[1] = Bb[1] + w * bxy.y;
        }
    }
}

// ------------------------------------------------------------ mixed form
// The mixed form's particle update: the CIC cell from the FP64 position, the
// eight weights and the gathered field in FP32 (fused multiply-adds), the
// magnetic field B = beta c (-E_y, E_x, 0) in FP32; then, in FP64 with fused
// multiply-adds, the beam -> reference frame rotation of R, E and B, the
// Boris kick, the half drift R += (c dt / 2) P / gamma (no unitless round
// trip) and the reference-frame update.  Results differ from the plain
// form's by rounding only (relative 1e-7 in E, 1e-16 in the FP64 steps).
__device__ __forceinline__ void cic_gather_f32(const float* __restrict__ E4, const int* n, const int* l, const float* d,
                                               float* Ef) {
    const int nx = n[0], nxy = n[0] * n[1];
    int zp[2];
    corner_planes(n, l[2], zp);
    const int b = l[0] + nx * l[1];
    const float u[3] = {1.0f - d[0], 1.0f - d[1], 1.0f - d[2]};
    float e0 = 0.0f, e1 = 0.0f, e2 = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int a0 = k & 1, a1 = (k >> 1) & 1, a2 = (k >> 2) & 1;
        const float w = (a0 ? d[0] : u[0]) * (a1 ? d[1] : u[1]) * (a2 ? d[2] : u[2]);
        const float4 a = __ldg(reinterpret_cast<const float4*>(E4) + (b + a0 + a1 * nx + zp[a2] * nxy));
        e0 = fmaf(w, a.x, e0);
        e1 = fmaf(w, a.y, e1);
        e2 = fmaf(w, a.z, e2);
    }
    Ef[0] = e0;
    Ef[1] = e1;
    Ef[2] = e2;
}
// returns false when the CIC stencil left the mesh
template <bool EXT>
__device__ __forceinline__ bool mixed_particle(const BunchConst& bc, const MeshConsts& m, const float* __restrict__ E4,
                                               const Trafo& b2r, const Trafo& upd, double betaC, const StepState* st,
                                               double* R, double* P) {
    int l[3];
    float d[3], e[3];
    const bool ok = cic_locate_fast(m.rhr, m.org, bc.n, R, l, d, bc.pz);
    cic_gather_f32(E4, bc.n, l, d, e);
    const float bc32 = (float)betaC;
    const double Eb[3] = {(double)e[0], (double)e[1], (double)e[2]};
    const double Bb[3] = {(double)(-bc32 * e[1]), (double)(bc32 * e[0]), 0.0};
    double X[3] = {R[0] - b2r.origin[0], R[1] - b2r.origin[1], R[2] - b2r.origin[2]};
    double Rr[3], Ef[3], Bf[3];
    matvec_fma(b2r.M, X, Rr);
    matvec_fma(b2r.M, Eb, Ef);
    matvec_fma(b2r.M, Bb, Bf);
    if (bc.bz_ext != 0.0) Bf[2] += bc.bz_ext;
    if constexpr (EXT) add_external_fields(bc.sol, bc.nsol, st->ref_to_lab_step, Rr, st->t_step + 0.5 * bc.dT, Ef, Bf);
    // Boris kick (BorisPusher.h:56-113)
    const double ke = bc.ke;
#pragma unroll
    for (int a = 0; a < 3; ++a) P[a] = fma(ke, Ef[a], P[a]);
    const double gamma = sqrt(fma(P[0], P[0], fma(P[1], P[1], fma(P[2], P[2], 1.0))));
    const double kt = bc.ktn / (gamma * bc.mass);
    const double t[3] = {kt * Bf[0], kt * Bf[1], kt * Bf[2]};
    double c[3], w[3];
    cross_fma(P, t, c);
    w[0] = P[0] + c[0];
    w[1] = P[1] + c[1];
    w[2] = P[2] + c[2];
    const double ks = 2.0 / fma(t[0], t[0], fma(t[1], t[1], fma(t[2], t[2], 1.0)));
    const double sv[3] = {ks * t[0], ks * t[1], ks * t[2]};
    cross_fma(w, sv, c);
#pragma unroll
    for (int a = 0; a < 3; ++a) P[a] = fma(ke, Ef[a], P[a] + c[a]);
    // half drift
    const double g = sqrt(fma(P[0], P[0], fma(P[1], P[1], fma(P[2], P[2], 1.0))));
    const double hv = (0.5 * bc.s_cdt) / g;
#pragma unroll
    for (int a = 0; a < 3; ++a) Rr[a] = fma(hv, P[a], Rr[a]);
    // reference-frame update
    double Y[3] = {Rr[0] - upd.origin[0], Rr[1] - upd.origin[1], Rr[2] - upd.origin[2]};
    matvec_fma(upd.M, Y, R);
    double Pu[3];
    matvec_fma(upd.M, P, Pu);
    P[0] = Pu[0];
    P[1] = Pu[1];
    P[2] = Pu[2];
    return ok;
}

// STAGED: the particle state streamed through shared memory (stream_chunks,
// dynamic shared memory sm); the arithmetic is the same either way.
template <typename T, bool BINNED = false, bool EXT = false, bool STAGED = false>
__device__ __forceinline__ void gather_body(const BunchConst& bc, double* __restrict__ x, double* __restrict__ y,
                                            double* __restrict__ z, double* __restrict__ px, double* __restrict__ py,
                                            double* __restrict__ pz, const T* __restrict__ E4, StepState* st,
                                            double* partials, unsigned* ticket, VB g, const double* __restrict__ F8 = nullptr,
                                            double* sm = nullptr) {
    __shared__ Trafo b2r_s, upd_s;
    __shared__ MeshConsts ms;
    __shared__ double betaC_s;
    __shared__ __align__(8) uint64_t bar[2];
    load_mesh_consts(ms, st);
    if (threadIdx.x == 0) {
        b2r_s = st->b2r;
        upd_s = st->upd;
        betaC_s = st->betaC;
        if constexpr (STAGED) {
            mbar_init(&bar[0], 1);
            mbar_init(&bar[1], 1);
            mbar_fence_init();
        }
    }
    __syncthreads();
    i128 acc[3] = {0, 0, 0};
    bool bad = false;
    // one particle: state X, P in, new state out to slot i
    auto one = [&](long long i, const double* X, const double* Pin) {
        double P[3] = {Pin[0], Pin[1], Pin[2]};
        double Ru[3], Pu[3];
        if constexpr (sizeof(T) == sizeof(float) && !BINNED) {
            double R[3] = {X[0], X[1], X[2]};
            if (!mixed_particle<EXT>(bc, *fresh(&ms), reinterpret_cast<const float*>(E4), *fresh(&b2r_s),
                                     *fresh(&upd_s), *fresh(&betaC_s), st, R, P))
                bad = true;
            Ru[0] = R[0], Ru[1] = R[1], Ru[2] = R[2];
            Pu[0] = P[0], Pu[1] = P[1], Pu[2] = P[2];
        } else {
            int l[3];
            double d[3];
            const MeshConsts* m = fresh(&ms);
            if (!cic_locate_r(m->hr, m->rhr, m->org, bc.n, X, l, d, bc.pz)) bad = true;
            double Eb[3], Bb[3];
            if constexpr (BINNED) {
                cic_gather8(F8, bc.n, l, d, Eb, Bb);
                Bb[2] = 0.0;
            } else {
                cic_gather(E4, bc.n, l, d, Eb);
                const double betaC = *fresh(&betaC_s);
                Bb[0] = 0.0 - betaC * Eb[1];
                Bb[1] = 0.0 + betaC * Eb[0];
                Bb[2] = 0.0;
            }
            double R[3], Ef[3], Bf[3];
            const Trafo* b2r = fresh(&b2r_s);
            trafo_transform_to(*b2r, X, R);
            trafo_rotate_to(*b2r, Eb, Ef);
            trafo_rotate_to(*b2r, Bb, Bf);
            if (bc.bz_ext != 0.0) Bf[2] += bc.bz_ext;
            // the beamline elements' fields at R, in the frame of the step's start
            if constexpr (EXT)
                add_external_fields(bc.sol, bc.nsol, st->ref_to_lab_step, R, st->t_step + 0.5 * bc.dT, Ef, Bf);
            kick_r(P, Ef, Bf, bc.ke, bc.ktn, bc.mass);
            push_r(R, P, bc.s_cdt, bc.rs_cdt);
            const Trafo* upd = fresh(&upd_s);
            trafo_transform_to(*upd, R, Ru);
            trafo_rotate_to(*upd, P, Pu);
        }
        x[i] = Ru[0];
        y[i] = Ru[1];
        z[i] = Ru[2];
        px[i] = Pu[0];
        py[i] = Pu[1];
        pz[i] = Pu[2];
        acc[0] += ex_from(Pu[0]);
        acc[1] += ex_from(Pu[1]);
        acc[2] += ex_from(Pu[2]);
    };
    if constexpr (STAGED) {
        const double* const src[6] = {x, y, z, px, py, pz};
        if (!stream_chunks<6>(src, bc.N, g, sm, bar, &st->err, [&](long long i, const double* q) { one(i, q, q + 3); }))
            return;
    } else {
        for (long long i = g.blk * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)g.nblk * blockDim.x) {
            const double X[3] = {x[i], y[i], z[i]};
            const double P[3] = {px[i], py[i], pz[i]};
            one(i, X, P);
        }
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
    i128* xpart = reinterpret_cast<i128*>(partials);
    block_sum_ex<3>(acc, xpart, g.blk);
    if (!last_block(ticket, g.nblk)) return;
    __shared__ double tot[3];
    __shared__ i128 ex[3];
    final_sum_ex<3>(xpart, g.nblk, tot, ex);
    __syncthreads();
    if (threadIdx.x == 0) {
        StepState& s = *st;
        if (bc.sharded) {  // this rank's momentum sums; k_finish_psum completes after the exchange
            for (int k = 0; k < 3; ++k) put_limbs(s.xlimbs + 4 * k, ex[k]);
        } else {
            s.psum[0] = tot[0];
            s.psum[1] = tot[1];
            s.psum[2] = tot[2];
            if (!derive_beam_frame(s, bc)) atomicOr(&s.err, kFlagFrame);
            s.step += 1;
        }
        *ticket = 0u;
    }
}
template <typename T, bool EXT = false>
__global__ void __launch_bounds__(kThreads, 3) k_gather_kick_push(BunchConst bc, double* __restrict__ x, double* __restrict__ y,
                                                                  double* __restrict__ z, double* __restrict__ px,
                                                                  double* __restrict__ py, double* __restrict__ pz,
                                                                  const T* __restrict__ E4, StepState* st, double* partials,
                                                                  unsigned* ticket) {
    gather_body<T, false, EXT>(bc, x, y, z, px, py, pz, E4, st, partials, ticket, vb_grid());
}
constexpr size_t kGatherSmem = 2 * 6 * kStreamChunk * sizeof(double);
template <typename T, bool EXT = false>
__global__ void __launch_bounds__(kThreads, 3) k_gather_staged(BunchConst bc, double* __restrict__ x, double* __restrict__ y,
                                                               double* __restrict__ z, double* __restrict__ px,
                                                               double* __restrict__ py, double* __restrict__ pz,
                                                               const T* __restrict__ E4, StepState* st, double* partials,
                                                               unsigned* ticket) {
    extern __shared__ __align__(16) double gather_sm[];
    gather_body<T, false, EXT, true>(bc, x, y, z, px, py, pz, E4, st, partials, ticket, vb_grid(), nullptr, gather_sm);
}
template <bool EXT = false>
__global__ void __launch_bounds__(kThreads, 3) k_gather_kick_push_bins(BunchConst bc, double* __restrict__ x,
                                                                       double* __restrict__ y, double* __restrict__ z,
                                                                       double* __restrict__ px, double* __restrict__ py,
                                                                       double* __restrict__ pz,
                                                                       const double* __restrict__ F8, StepState* st,
                                                                       double* partials, unsigned* ticket) {
    gather_body<double, true, EXT>(bc, x, y, z, px, py, pz, nullptr, st, partials, ticket, vb_grid(), F8);
}

// Fields only (PartBunch::computeSelfFields output): Ef, Bf in the beam frame,
// AoS (x, y, z per particle).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_gather_fields(BunchConst bc, const double* __restrict__ x,
                                                            const double* __restrict__ y, const double* __restrict__ z,
                                                            const T* __restrict__ E4, StepState* st, double* __restrict__ Ef,
                                                            double* __restrict__ Bf) {
    __shared__ double hr[3], rhr[3], org[3], betaC;
    if (threadIdx.x < 3) {
        hr[threadIdx.x] = st->hr[threadIdx.x];
        rhr[threadIdx.x] = st->rhr[threadIdx.x];
        org[threadIdx.x] = st->origin[threadIdx.x];
    }
    if (threadIdx.x == 0) betaC = st->betaC;
    __syncthreads();
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        double X[3] = {x[i], y[i], z[i]};
        int l[3];
        double d[3];
        if (!cic_locate_r(hr, rhr, org, bc.n, X, l, d, bc.pz)) bad = true;
        double E[3];
        cic_gather(E4, bc.n, l, d, E);
        Ef[3 * i + 0] = E[0];
        Ef[3 * i + 1] = E[1];
        Ef[3 * i + 2] = E[2];
        Bf[3 * i + 0] = 0.0 - betaC * E[1];
        Bf[3 * i + 1] = 0.0 + betaC * E[0];
        Bf[3 * i + 2] = 0.0;
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
}
__global__ void __launch_bounds__(kThreads) k_gather_fields_bins(BunchConst bc, const double* __restrict__ x,
                                                                 const double* __restrict__ y,
                                                                 const double* __restrict__ z,
                                                                 const double* __restrict__ F8, StepState* st,
                                                                 double* __restrict__ Ef, double* __restrict__ Bf) {
    __shared__ double hr[3], rhr[3], org[3];
    if (threadIdx.x < 3) {
        hr[threadIdx.x] = st->hr[threadIdx.x];
        rhr[threadIdx.x] = st->rhr[threadIdx.x];
        org[threadIdx.x] = st->origin[threadIdx.x];
    }
    __syncthreads();
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        double X[3] = {x[i], y[i], z[i]};
        int l[3];
        double d[3];
        if (!cic_locate_r(hr, rhr, org, bc.n, X, l, d)) bad = true;
        double E[3], B[2];
        cic_gather8(F8, bc.n, l, d, E, B);
        Ef[3 * i + 0] = E[0];
        Ef[3 * i + 1] = E[1];
        Ef[3 * i + 2] = E[2];
        Bf[3 * i + 0] = B[0];
        Bf[3 * i + 1] = B[1];
        Bf[3 * i + 2] = 0.0;
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
}

__global__ void __launch_bounds__(kThreads) k_aos_to_soa_by_id(const double* __restrict__ aos,
                                                               const uint32_t* __restrict__ id, double* __restrict__ a,
                                                               double* __restrict__ b, double* __restrict__ c,
                                                               long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const size_t q = 3 * (size_t)id[i];
        a[i] = aos[q + 0];
        b[i] = aos[q + 1];
        c[i] = aos[q + 2];
    }
}

__global__ void __launch_bounds__(kThreads) k_aos_to_soa(const double* __restrict__ aos, double* __restrict__ a,
                                                         double* __restrict__ b, double* __restrict__ c, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        a[i] = aos[3 * i + 0];
        b[i] = aos[3 * i + 1];
        c[i] = aos[3 * i + 2];
    }
}

__global__ void __launch_bounds__(kThreads) k_soa_to_aos(const double* __restrict__ a, const double* __restrict__ b,
                                                         const double* __restrict__ c, double* __restrict__ aos, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        aos[3 * i + 0] = a[i];
        aos[3 * i + 1] = b[i];
        aos[3 * i + 2] = c[i];
    }
}

// Particle p of the cell-sorted order: copy slot sval[p] to position p of the
// staging buffers (six coordinate arrays and the original index).
__global__ void __launch_bounds__(kThreads) k_reorder(const uint32_t* __restrict__ sval, const double* __restrict__ x,
                                                      const double* __restrict__ y, const double* __restrict__ z,
                                                      const double* __restrict__ px, const double* __restrict__ py,
                                                      const double* __restrict__ pz, const uint32_t* __restrict__ id,
                                                      double* __restrict__ sa, double* __restrict__ sb,
                                                      uint32_t* __restrict__ sid, long long n) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const uint32_t q = sval[p];
        sa[p] = x[q];
        sa[n + p] = y[q];
        sa[2 * n + p] = z[q];
        sb[p] = px[q];
        sb[n + p] = py[q];
        sb[2 * n + p] = pz[q];
        sid[p] = id[q];
    }
}

__global__ void __launch_bounds__(kThreads) k_iota(uint32_t* __restrict__ id, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        id[i] = (uint32_t)i;
}

// slot order -> original particle order, AoS
__global__ void __launch_bounds__(kThreads) k_soa_to_aos_by_id(const double* __restrict__ a, const double* __restrict__ b,
                                                               const double* __restrict__ c, const uint32_t* __restrict__ id,
                                                               double* __restrict__ aos, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const long long o = id[i];
        aos[3 * o + 0] = a[i];
        aos[3 * o + 1] = b[i];
        aos[3 * o + 2] = c[i];
    }
}

template <typename TI, typename TO>
__global__ void __launch_bounds__(kThreads) k_convert(const TI* __restrict__ in, TO* __restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = (TO)in[i];
}

inline int grid_for(long long work, int cap) {
    long long g = (work + kThreads - 1) / kThreads;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (int)g;
}

// ------------------------------------------------------------ batched launches
// One kernel over many bunches: block i takes work item work[i] = (bunch,
// block, -, blocks of that bunch) and runs the same body as the single-bunch
// kernel on the bunch's buffers (tab[bunch], a device copy of its DevBunch).
template <bool DRIFT, bool MIXED = false>
__global__ void __launch_bounds__(kThreads, 3) k_drift_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    drift_body<DRIFT, MIXED>(d.bc, d.x, d.y, d.z, d.px, d.py, d.pz, d.st, d.partials, d.ticket, VB{w.y, w.w});
}

template <bool STATS>
__global__ void __launch_bounds__(kThreads) k_reduce_state_batch(const DevBunch* __restrict__ tab,
                                                                 const int4* __restrict__ work, int nitems, bool init_frame) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    reduce_state_body<STATS>(d.bc, d.x, d.y, d.z, d.px, d.py, d.pz, d.st, d.partials, d.ticket, init_frame,
                             VB{w.y, w.w});
}

template <int NT, bool MIXED = false>
__global__ void __launch_bounds__(NT) k_deposit_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    if constexpr (MIXED)
        deposit_mixed_body<false>(d.bc, d.x, d.y, d.z, d.st, d.nacc, VB{w.y, w.w});
    else
        deposit_pairs_body(d.bc, d.x, d.y, d.z, d.st, d.nacc, VB{w.y, w.w});
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_assemble_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    assemble_body<T>(d.bc, d.st, d.nacc, (T*)d.rho, VB{w.y, w.w}, d.dep_weights != 0);
}

__global__ void k_advance_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    advance_reference_body(d.bc, d.st, VB{w.y, w.w});
}

__global__ void __launch_bounds__(kThreads) k_igf_tmp_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    if (d.precision == 0)
        igf_tmp_body<true>(d.bc.n[0], d.bc.n[1], d.bc.n[2], d.st, d.gtmp, VB{w.y, w.w});
    else
        igf_tmp_body<false>(d.bc.n[0], d.bc.n[1], d.bc.n[2], d.st, d.gtmp, VB{w.y, w.w});
}

__global__ void __launch_bounds__(kThreads) k_igf_G_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    igf_G_body(d.bc.n[0], d.bc.n[1], d.bc.n[2], d.gtmp, d.gline, VB{w.y, w.w});
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_grad_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    grad_body<T>(d.bc, d.st, d.phi, (T*)d.E4, VB{w.y, w.w});
}

template <typename T>
__global__ void __launch_bounds__(kThreads, 3) k_gather_batch(const DevBunch* __restrict__ tab, const int4* __restrict__ work, int nitems) {
    const int4 w = resolve_block(work, nitems);
    const DevBunch& d = tab[w.x];
    gather_body<T>(d.bc, d.x, d.y, d.z, d.px, d.py, d.pz, (const T*)d.E4, d.st, d.partials, d.ticket, VB{w.y, w.w});
}

}  // namespace

void launch_batch(int kind, int precision, int threads, const DevBunch* tab, const int4* work, int nitems, int nblocks,
                  cudaStream_t s) {
    if (nblocks <= 0 || nitems <= 0) return;
    const bool f64 = precision == 0;
    switch (kind) {
        case kBatchDrift:
            if (f64)
                k_drift_batch<true><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            else
                k_drift_batch<true, true><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            break;
        case kBatchPsum: k_reduce_state_batch<false><<<nblocks, kThreads, 0, s>>>(tab, work, nitems, true); break;
        case kBatchStats: k_reduce_state_batch<true><<<nblocks, kThreads, 0, s>>>(tab, work, nitems, false); break;
        case kBatchDeposit:
            if (threads == 128)
                (f64 ? k_deposit_batch<128> : k_deposit_batch<128, true>)<<<nblocks, 128, 0, s>>>(tab, work, nitems);
            else if (threads == 512)
                (f64 ? k_deposit_batch<512> : k_deposit_batch<512, true>)<<<nblocks, 512, 0, s>>>(tab, work, nitems);
            else
                (f64 ? k_deposit_batch<256> : k_deposit_batch<256, true>)<<<nblocks, 256, 0, s>>>(tab, work, nitems);
            break;
        case kBatchAssemble:
            if (f64)
                k_assemble_batch<double><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            else
                k_assemble_batch<float><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            break;
        case kBatchAdvance: k_advance_batch<<<nblocks, 32, 0, s>>>(tab, work, nitems); break;
        case kBatchIgfTmp: k_igf_tmp_batch<<<nblocks, kThreads, 0, s>>>(tab, work, nitems); break;
        case kBatchIgfG: k_igf_G_batch<<<nblocks, kThreads, 0, s>>>(tab, work, nitems); break;
        case kBatchGrad:
            if (f64)
                k_grad_batch<double><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            else
                k_grad_batch<float><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            break;
        case kBatchGather:
            if (f64)
                k_gather_batch<double><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            else
                k_gather_batch<float><<<nblocks, kThreads, 0, s>>>(tab, work, nitems);
            break;
        default: break;
    }
}

int particle_grid(const DevBunch& b) { return b.red_blocks; }

#ifndef SC_PARTICLE_WAVES
#define SC_PARTICLE_WAVES 1
#endif

constexpr int kMaxCachedDevices = 64;

// Resident blocks of kThreads on the whole current device for one kernel
// (the occupancy query runs once per device and kernel, outside stream
// capture: contexts call prime_particle_grids when they are created).  The
// cache is keyed by the device too, since devices may differ in SM count.
int resident_blocks(const void* kernel, size_t smem = 0) {
    static std::mutex mu;
    static std::unordered_map<const void*, int> cache[kMaxCachedDevices];
    int dev = 0, nsm = 0, k = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    std::unordered_map<const void*, int>* c = (dev >= 0 && dev < kMaxCachedDevices) ? &cache[dev] : nullptr;
    if (c) {
        auto it = c->find(kernel);
        if (it != c->end()) return it->second;
    }
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || nsm <= 0) nsm = 148;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&k, kernel, kThreads, smem) != cudaSuccess || k < 1) k = 1;
    cudaGetLastError();
    if (!c) return k * nsm;
    return c->emplace(kernel, k * nsm).first->second;
}

// Blocks for a particle loop (grid-stride, one reduction per block): the
// blocks the SMs hold at once, SC_PARTICLE_WAVES times, so each block loops
// over several particles and its set-up and reduction are paid once per
// resident block; never more than b.red_blocks (the partials' size).
template <typename K>
int wave_grid(K kernel, const DevBunch& b, size_t smem = 0) {
    if (SC_PARTICLE_WAVES <= 0) return b.red_blocks;
    const int blocks = resident_blocks((const void*)kernel, smem) * SC_PARTICLE_WAVES;
    return blocks < b.red_blocks ? blocks : b.red_blocks;
}

// The gather streams the particle state through shared memory with bulk
// copies (default); SCGPU_STREAM=0 selects the direct-load kernel (same bits).
bool stream_particles() {
    static const bool on = [] {
        const char* e = std::getenv("SCGPU_STREAM");
        return !(e && std::string(e) == "0");
    }();
    return on;
}


void prime_particle_grids() {
    cudaFuncSetAttribute(k_gather_staged<double, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGatherSmem);
    cudaFuncSetAttribute(k_gather_staged<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGatherSmem);
    cudaFuncSetAttribute(k_gather_staged<float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGatherSmem);
    cudaFuncSetAttribute(k_gather_staged<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGatherSmem);
    const void* kernels[] = {(const void*)k_drift_to_beam<true>,
                             (const void*)k_drift_to_beam<true, true>,
                             (const void*)k_drift_to_beam<false>,
                             (const void*)k_deposit<false>,
                             (const void*)k_deposit<true>,
                             (const void*)k_deposit_mixed<false>,
                             (const void*)k_deposit_mixed<true>,
                             (const void*)k_deposit_bins,
                             (const void*)k_gather_kick_push<double, false>,
                             (const void*)k_gather_kick_push<double, true>,
                             (const void*)k_gather_kick_push<float, false>,
                             (const void*)k_gather_kick_push<float, true>,
                             (const void*)k_gather_kick_push_bins<false>,
                             (const void*)k_gather_kick_push_bins<true>};
    for (const void* k : kernels) resident_blocks(k);
    const void* staged[] = {(const void*)k_gather_staged<double, false>, (const void*)k_gather_staged<double, true>,
                            (const void*)k_gather_staged<float, false>, (const void*)k_gather_staged<float, true>};
    for (const void* k : staged) resident_blocks(k, kGatherSmem);
}

void launch_reduce_state(const DevBunch& b, bool init_frame, cudaStream_t s) {
    k_reduce_state<false><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.st, b.partials,
                                                           b.ticket, init_frame);
}

void launch_drift_to_beam(const DevBunch& b, bool drift, cudaStream_t s, bool mixed) {
    auto k = !drift ? k_drift_to_beam<false> : mixed ? k_drift_to_beam<true, true> : k_drift_to_beam<true>;
    k<<<wave_grid(k, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.st, b.partials, b.ticket);
}

void launch_advance_reference(const DevBunch& b, cudaStream_t s) { k_advance_reference<<<1, 32, 0, s>>>(b.bc, b.st); }

void launch_cell_keys(const DevBunch& b, int digit_bits, cudaStream_t s) {
    (void)digit_bits;
    k_cell_keys<<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.st, b.keys, b.vals_alt, b.hist);
}

void launch_deposit(const DevBunch& b, cudaStream_t s) {
    if (b.dep_weights) {
        auto k = b.bc.pz ? k_deposit_mixed<true> : k_deposit_mixed<false>;
        k<<<wave_grid(k, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.st, b.nacc);
    } else if (b.bc.pz)
        k_deposit<true><<<wave_grid(k_deposit<true>, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.st, b.nacc);
    else
        k_deposit<false><<<wave_grid(k_deposit<false>, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.st, b.nacc);
}

void launch_assemble_rho(const DevBunch& b, cudaStream_t s) {
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    const int g = grid_for(M, 148 * 16);
    if (b.precision == 0)
        k_assemble_rho<double><<<g, kThreads, 0, s>>>(b.bc, b.st, b.nacc, (double*)b.rho, b.dep_weights);
    else
        k_assemble_rho<float><<<g, kThreads, 0, s>>>(b.bc, b.st, b.nacc, (float*)b.rho, b.dep_weights);
}

void launch_igf(const DevBunch& b, const double* hr_host, cudaStream_t s) {
    (void)hr_host;
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long T3 = (long long)(n0 + 2) * (n1 + 2) * (n2 + 2);
    const long long G3 = (long long)(n0 + 1) * (n1 + 1) * (n2 + 1);
    if (b.precision == 0)
        k_igf_tmp<true><<<grid_for(T3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.st, b.gtmp);
    else
        k_igf_tmp<false><<<grid_for(T3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.st, b.gtmp);
    k_igf_G<<<grid_for(G3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.gtmp, b.gline);
}

// The antiderivative alone (b.gtmp): launch_green_transform_from_tmp forms G
// from it inside its first cosine transform.
void launch_igf_tmp(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long T3 = (long long)(n0 + 2) * (n1 + 2) * (n2 + 2);
    if (b.precision == 0)
        k_igf_tmp<true><<<grid_for(T3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.st, b.gtmp);
    else
        k_igf_tmp<false><<<grid_for(T3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.st, b.gtmp);
}

void launch_grad(const DevBunch& b, cudaStream_t s) {
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    const int g = grid_for(M, 148 * 16);
    if (b.precision == 0)
        k_grad<double><<<g, kThreads, 0, s>>>(b.bc, b.st, b.phi, (double*)b.E4);
    else
        k_grad<float><<<g, kThreads, 0, s>>>(b.bc, b.st, b.phi, (float*)b.E4);
}

void launch_gather_kick_push(const DevBunch& b, bool stats, cudaStream_t s) {
    const bool ext = b.bc.nsol > 0;
    if (stream_particles()) {
        if (b.precision == 0) {
            auto k = ext ? k_gather_staged<double, true> : k_gather_staged<double, false>;
            k<<<wave_grid(k, b, kGatherSmem), kThreads, kGatherSmem, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz,
                                                                           (const double*)b.E4, b.st, b.partials,
                                                                           b.ticket);
        } else {
            auto k = ext ? k_gather_staged<float, true> : k_gather_staged<float, false>;
            k<<<wave_grid(k, b, kGatherSmem), kThreads, kGatherSmem, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz,
                                                                           (const float*)b.E4, b.st, b.partials,
                                                                           b.ticket);
        }
        if (stats) launch_reduce_stats(b, s);
        return;
    }
    if (b.precision == 0) {
        auto k = ext ? k_gather_kick_push<double, true> : k_gather_kick_push<double, false>;
        k<<<wave_grid(k, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, (const double*)b.E4, b.st,
                                               b.partials, b.ticket);
    } else {
        auto k = ext ? k_gather_kick_push<float, true> : k_gather_kick_push<float, false>;
        k<<<wave_grid(k, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, (const float*)b.E4, b.st,
                                               b.partials, b.ticket);
    }
    if (stats) launch_reduce_stats(b, s);
}

void launch_gather_fields(const DevBunch& b, cudaStream_t s) {
    if (b.precision == 0)
        k_gather_fields<double><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, (const double*)b.E4, b.st, b.Ef, b.Bf);
    else
        k_gather_fields<float><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, (const float*)b.E4, b.st, b.Ef, b.Bf);
}

void launch_finish_mesh(const DevBunch& b, cudaStream_t s) { k_finish_mesh<<<1, 32, 0, s>>>(b.bc, b.st); }
void launch_finish_psum(const DevBunch& b, bool frame, bool advance, cudaStream_t s) {
    k_finish_psum<<<1, 32, 0, s>>>(b.bc, b.st, frame ? 1 : 0, advance ? 1 : 0);
}
void launch_finish_stats(const DevBunch& b, cudaStream_t s) { k_finish_stats<<<1, 32, 0, s>>>(b.st); }

constexpr int kBinGammaBlocks = 296;

void launch_bin_gammas(const DevBunch& b, cudaStream_t s) {
    const int g = b.red_blocks < kBinGammaBlocks ? b.red_blocks : kBinGammaBlocks;
    k_bin_gammas<<<g, kThreads, 0, s>>>(b.bc, b.px, b.py, b.pz, b.bin, b.nbins, b.st, b.bst, b.bin_partials, b.ticket);
}

void launch_deposit_bins(const DevBunch& b, cudaStream_t s) {
    k_deposit_bins<<<wave_grid(k_deposit_bins, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.bin, b.nactive, b.st,
                                                                      b.nacc_bins);
}

void launch_grad_acc(const DevBunch& v, const double* phi_img, cudaStream_t s) {
    const long long M = (long long)v.bc.n[0] * v.bc.n[1] * v.bc.n[2];
    const int g = grid_for(M, 148 * 16);
    k_grad_acc<<<g, kThreads, 0, s>>>(v.bc, v.st, v.phi, phi_img, v.F8);
}

void launch_gather_kick_push_bins(const DevBunch& b, bool stats, cudaStream_t s) {
    auto k = b.bc.nsol > 0 ? k_gather_kick_push_bins<true> : k_gather_kick_push_bins<false>;
    k<<<wave_grid(k, b), kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.F8, b.st, b.partials, b.ticket);
    if (stats) launch_reduce_stats(b, s);
}

void launch_gather_fields_bins(const DevBunch& b, cudaStream_t s) {
    k_gather_fields_bins<<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.F8, b.st, b.Ef, b.Bf);
}

void launch_bounds(const DevBunch& b, double* out6, cudaStream_t s) {
    k_bounds<<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.partials, b.ticket, out6);
}

void launch_find_id(const DevBunch& b, uint32_t target, double* out6, cudaStream_t s) {
    k_find_id<<<grid_for(b.bc.N, 148 * 16), kThreads, 0, s>>>(b.id, b.bc.N, target, b.x, b.y, b.z, b.px, b.py, b.pz, out6);
}

void launch_bins_by_id(const int* host_order, const uint32_t* id, int* bin, long long n, cudaStream_t s) {
    k_bins_by_id<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(host_order, id, bin, n);
}

void launch_permute_bins(const DevBunch& b, cudaStream_t s) {
    const long long n = b.bc.N;
    k_permute_i32<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(b.vals, b.bin, b.bin_alt, n);
    cudaMemcpyAsync(b.bin, b.bin_alt, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, s);
}

void launch_igf_image(const DevBunch& b, cudaStream_t s) {
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long T3 = (long long)(n0 + 2) * (n1 + 2) * (n2 + 2);
    const long long GI = (long long)(n0 + 1) * (n1 + 1) * (2 * n2);
    k_igf_tmp_img<<<grid_for(2 * T3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.st, b.gtmp_img);
    k_igf_G_img<<<grid_for(GI, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.gtmp_img, b.gimg);
}

void launch_aos_to_soa_by_id(const double* aos, const uint32_t* id, double* a, double* b, double* c, long long n,
                             cudaStream_t s) {
    k_aos_to_soa_by_id<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(aos, id, a, b, c, n);
}

void launch_aos_to_soa(const double* aos, double* a, double* b, double* c, long long n, cudaStream_t s) {
    k_aos_to_soa<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(aos, a, b, c, n);
}

void launch_soa_to_aos(const double* a, const double* b, const double* c, double* aos, long long n, cudaStream_t s) {
    k_soa_to_aos<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(a, b, c, aos, n);
}

// Puts the particle arrays in cell order (the order of the last counting
// sort); b.Ef / b.Bf / b.keys_alt are the staging buffers.
void launch_reorder(const DevBunch& b, cudaStream_t s) {
    const long long n = b.bc.N;
    k_reorder<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(b.vals, b.x, b.y, b.z, b.px, b.py, b.pz, b.id, b.Ef, b.Bf,
                                                         b.keys_alt, n);
    const size_t d = (size_t)n * sizeof(double);
    cudaMemcpyAsync(b.x, b.Ef, d, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.y, b.Ef + n, d, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.z, b.Ef + 2 * n, d, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.px, b.Bf, d, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.py, b.Bf + n, d, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.pz, b.Bf + 2 * n, d, cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(b.id, b.keys_alt, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
}

void launch_iota(uint32_t* id, long long n, cudaStream_t s) { k_iota<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(id, n); }

void launch_soa_to_aos_by_id(const double* a, const double* b, const double* c, const uint32_t* id, double* aos,
                             long long n, cudaStream_t s) {
    k_soa_to_aos_by_id<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(a, b, c, id, aos, n);
}

void launch_f64_to_f32(const double* in, float* out, long long n, cudaStream_t s) {
    k_convert<double, float><<<grid_for(n, 148 * 16), kThreads, 0, s>>>(in, out, n);
}

void launch_f32_to_f64(const float* in, double* out, long long n, cudaStream_t s) {
    k_convert<float, double><<<grid_for(n, 148 * 16), kThreads, 0, s>>>(in, out, n);
}

void launch_reduce_stats(const DevBunch& b, cudaStream_t s) {
    k_reduce_state<true><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.st, b.partials,
                                                          b.ticket, false);
}

}  // namespace sc
