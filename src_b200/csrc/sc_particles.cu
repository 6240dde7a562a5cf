// sc_particles.cu -- particle-side kernels of the space-charge step.
//
// Compiled with -fmad=false: every per-particle expression rounds like the
// reference's CPU code (push, kick, frame transforms, CIC weights).
//
//   k_reduce_state       momentum sums (+ beam statistics) and the beam frame
//   k_drift_to_beam      half drift, reference -> beam frame, bounds, mesh
//   k_cell_keys          CIC lower-grid-point cell key + radix digit histogram
//   k_deposit_windows    warp-level segmented reduction over cell-sorted particles
//   k_deposit_resolve    joins cells whose particles span several warp windows
//   k_assemble_rho       corner sums -> charge density on the n^3 cell field
//   k_igf_tmp, k_igf_G   integrated Green's function (FFTPoissonSolver.cpp:459-522)
//   k_grad               -Grad phi (UniformCartesian.hpp:2129-2203), boost scaling
//   k_gather_kick_push   CIC gather, B from E, back to the reference frame, Boris
//                        kick, half drift, reference-particle frame update
#include <cstdio>

#include "sc_internal.h"

namespace sc {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr unsigned kFull = 0xffffffffu;

// ------------------------------------------------------------ reductions
// Deterministic block sum of NV values per thread into partials[block][NV].
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* __restrict__ partials) {
    __shared__ double sm[NV][kWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
#pragma unroll
        for (int k = 0; k < NV; ++k) v[k] += __shfl_down_sync(kFull, v[k], off);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sm[k][warp] = v[k];
    __syncthreads();
    for (int k = threadIdx.x; k < NV; k += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kWarps; ++w) s += sm[k][w];
        partials[(size_t)blockIdx.x * NV + k] = s;
    }
}

// Last-block-done: true in exactly one block, after every block's partials
// are visible.  The caller resets the ticket.
__device__ __forceinline__ bool last_block(unsigned* ticket) {
    __shared__ bool am_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) am_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    __syncthreads();
    return am_last;
}

// Sum of column k over nb block partials, in a fixed order; result in lane 0
// of the warp that handles k.  out[k] receives the totals.
template <int NV>
__device__ __forceinline__ void final_sum(const double* partials, int nb, double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = warp; k < NV; k += kWarps) {
        double s = 0.0;
        for (int b = lane; b < nb; b += 32) s += __ldcg(partials + (size_t)b * NV + k);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(kFull, s, off);
        if (lane == 0) out[k] = s;
    }
}

// moments in OPAL's order (x, px, y, py, z, pz), PartBunchBase.hpp:2185-2259,
// plus sum of gamma (:1588-1593) as value 27.
__device__ __forceinline__ void accumulate_moments(double (&m)[28], const double* R, const double* P) {
    double part[6] = {R[0], P[0], R[1], P[1], R[2], P[2]};
    int l = 6;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        m[i] += part[i];
#pragma unroll
        for (int j = 0; j <= i; ++j) m[l++] += part[i] * part[j];
    }
    m[27] += sqrt(1.0 + dot3(P, P));
}

// ------------------------------------------------------------ state reduction
template <bool STATS>
__global__ void __launch_bounds__(kThreads) k_reduce_state(BunchConst bc, const double* __restrict__ x,
                                                           const double* __restrict__ y, const double* __restrict__ z,
                                                           const double* __restrict__ px, const double* __restrict__ py,
                                                           const double* __restrict__ pz, StepState* st,
                                                           double* partials, unsigned* ticket, bool init_frame) {
    constexpr int NV = STATS ? 28 : 3;
    double v[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        double P[3] = {px[i], py[i], pz[i]};
        if constexpr (STATS) {
            double R[3] = {x[i], y[i], z[i]};
            double m[28];
            for (int k = 0; k < 28; ++k) m[k] = v[k];
            accumulate_moments(m, R, P);
            for (int k = 0; k < 28; ++k) v[k] = m[k];
        } else {
            v[0] += P[0];
            v[1] += P[1];
            v[2] += P[2];
        }
    }
    block_sum<NV>(v, partials);
    if (!last_block(ticket)) return;
    __shared__ double tot[NV];
    final_sum<NV>(partials, gridDim.x, tot);
    __syncthreads();
    if (threadIdx.x == 0) {
        if constexpr (STATS) {
            for (int k = 0; k < 27; ++k) st->moments[k] = tot[k];
            st->gsum = tot[27];
            st->psum[0] = tot[1];
            st->psum[1] = tot[3];
            st->psum[2] = tot[5];
        } else {
            st->psum[0] = tot[0];
            st->psum[1] = tot[1];
            st->psum[2] = tot[2];
        }
        if (init_frame && !derive_beam_frame(*st, bc)) atomicOr(&st->err, kFlagFrame);
        *ticket = 0u;
    }
}

// ------------------------------------------------------------ drift + frame
template <bool DRIFT>
__global__ void __launch_bounds__(kThreads) k_drift_to_beam(BunchConst bc, double* __restrict__ x, double* __restrict__ y,
                                                            double* __restrict__ z, const double* __restrict__ px,
                                                            const double* __restrict__ py, const double* __restrict__ pz,
                                                            StepState* st, double* partials, unsigned* ticket,
                                                            bool advance_ref) {
    __shared__ Trafo r2b;
    if (threadIdx.x == 0) r2b = st->r2b;
    __syncthreads();
    double v[6] = {INFINITY, INFINITY, INFINITY, INFINITY, INFINITY, INFINITY};  // min x,y,z, -max x,y,z
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        double R[3] = {x[i], y[i], z[i]};
        if constexpr (DRIFT) {
            double P[3] = {px[i], py[i], pz[i]};
            push_one(R, P, bc.dT);
            double b[3];
            trafo_transform_to(r2b, R, b);
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
    // min is exact and order-independent
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
    if (!last_block(ticket)) return;
    if (threadIdx.x == 0) {
        double m[6];
        for (int k = 0; k < 6; ++k) m[k] = INFINITY;
        for (unsigned b = 0; b < gridDim.x; ++b)
            for (int k = 0; k < 6; ++k) m[k] = fmin(m[k], __ldcg(partials + (size_t)b * 6 + k));
        StepState& s = *st;
        for (int k = 0; k < 3; ++k) {
            s.bmin[k] = m[k];
            s.bmax[k] = -m[3 + k];
        }
        if (!derive_mesh(s, bc)) atomicOr(&s.err, kFlagMesh);
        // Q *= dt; scatter; Q /= dt  (PartBunch.cpp:493-495)
        s.qdt = s.Q * bc.dT;
        s.Q = s.qdt / bc.dT;
        s.gen += 1u;
        if (s.gen == 0u) s.gen = 1u;
        if (advance_ref && !advance_reference(s, bc)) atomicOr(&s.err, kFlagFrame);
        *ticket = 0u;
    }
}

// ------------------------------------------------------------ cell keys
// key = lgp_x + n0 * (lgp_y + n1 * lgp_z); one block per sort tile, with the
// tile's digit histogram for the first radix pass.
__global__ void __launch_bounds__(kThreads) k_cell_keys(BunchConst bc, const double* __restrict__ x,
                                                        const double* __restrict__ y, const double* __restrict__ z,
                                                        StepState* st, uint32_t* __restrict__ keys, int* __restrict__ hist,
                                                        int tiles, int tile_elems, int digit_bits) {
    extern __shared__ int h[];
    const int bins = 1 << digit_bits;
    for (int d = threadIdx.x; d < bins; d += blockDim.x) h[d] = 0;
    __shared__ double hr[3], org[3];
    if (threadIdx.x < 3) {
        hr[threadIdx.x] = st->hr[threadIdx.x];
        org[threadIdx.x] = st->origin[threadIdx.x];
    }
    __syncthreads();
    const long long begin = (long long)blockIdx.x * tile_elems;
    long long end = begin + tile_elems;
    if (end > bc.N) end = bc.N;
    bool bad = false;
    for (long long i = begin + threadIdx.x; i < end; i += blockDim.x) {
        double X[3] = {x[i], y[i], z[i]};
        int l[3];
        double d[3];
        if (!cic_locate(hr, org, bc.n, X, l, d)) bad = true;
        uint32_t key = (uint32_t)l[0] + (uint32_t)bc.n[0] * ((uint32_t)l[1] + (uint32_t)bc.n[1] * (uint32_t)l[2]);
        keys[i] = key;
        atomicAdd(&h[key & (bins - 1)], 1);
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
    __syncthreads();
    for (int d = threadIdx.x; d < bins; d += blockDim.x) hist[(size_t)d * tiles + blockIdx.x] = h[d];
}

// ------------------------------------------------------------ deposit
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

enum : int { kWinFirst = 1, kWinLast = 2, kWinMid = 4 };

// One warp per window of 32 consecutive cell-sorted particles.  A segmented
// inclusive scan over the lanes (fixed Hillis-Steele tree, no atomics) sums
// the 8 corner charges of every cell present in the window.  Cells that lie
// wholly inside the window are written directly; the pieces of cells that
// continue into a neighbouring window go to the window's carry slots.
__global__ void __launch_bounds__(kThreads) k_deposit_windows(BunchConst bc, const uint32_t* __restrict__ skey,
                                                              const uint32_t* __restrict__ sval,
                                                              const double* __restrict__ x, const double* __restrict__ y,
                                                              const double* __restrict__ z, const StepState* __restrict__ st,
                                                              double* __restrict__ seg, uint32_t* __restrict__ stamp,
                                                              double* __restrict__ carry_first, double* __restrict__ carry_last,
                                                              int* __restrict__ wflag, long long nwin) {
    const int lane = threadIdx.x & 31;
    const long long w = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
    if (w >= nwin) return;
    const long long pos = w * 32 + lane;
    const bool valid = pos < bc.N;
    const uint32_t key = valid ? skey[pos] : 0xffffffffu;
    double v[8];
    if (valid) {
        const uint32_t p = sval[pos];
        double X[3] = {x[p], y[p], z[p]};
        int l[3];
        double d[3];
        cic_locate(st->hr, st->origin, bc.n, X, l, d);
        cic_charge(d, st->qdt, v);
    } else {
#pragma unroll
        for (int c = 0; c < 8; ++c) v[c] = 0.0;
    }
    const uint32_t kprev = __shfl_up_sync(kFull, key, 1);
    const uint32_t knext = __shfl_down_sync(kFull, key, 1);
    const bool head = (lane == 0) || (kprev != key);
    const bool tail = (lane == 31) || (knext != key);
    const unsigned heads = __ballot_sync(kFull, head);
    const int hd = 31 - __clz(heads & (lane == 31 ? kFull : ((2u << lane) - 1u)));
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            const double t = __shfl_up_sync(kFull, v[c], off);
            if (lane - off >= hd) v[c] += t;
        }
    }
    // does the segment of lane 0 start before this window / lane 31's continue after?
    uint32_t before = 0xfffffffeu, after = 0xfffffffeu;
    if (lane == 0 && w > 0) before = skey[pos - 1];
    if (lane == 31 && pos + 1 < bc.N) after = skey[pos + 1];
    before = __shfl_sync(kFull, before, 0);
    after = __shfl_sync(kFull, after, 31);
    const uint32_t key0 = __shfl_sync(kFull, key, 0);
    const bool cont_before = (before == key0);  // lane 0's cell started earlier
    const bool cont_after = (after == key) && lane == 31 && valid;
    const unsigned gen = st->gen;
    int flag = 0;
    if (valid && tail) {
        const bool starts_here = (hd > 0) || !cont_before;
        const bool ends_here = !cont_after;
        if (starts_here && ends_here) {
            double* s = seg + (size_t)key * 8;
#pragma unroll
            for (int c = 0; c < 8; ++c) s[c] = v[c];
            stamp[key] = gen;
        } else if (!starts_here && ends_here) {
            flag = kWinFirst;
#pragma unroll
            for (int c = 0; c < 8; ++c) carry_first[(size_t)w * 8 + c] = v[c];
        } else if (starts_here && !ends_here) {
            flag = kWinLast;
#pragma unroll
            for (int c = 0; c < 8; ++c) carry_last[(size_t)w * 8 + c] = v[c];
        } else {
            flag = kWinMid;
#pragma unroll
            for (int c = 0; c < 8; ++c) carry_first[(size_t)w * 8 + c] = v[c];
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) flag |= __shfl_xor_sync(kFull, flag, off);
    if (lane == 0) wflag[w] = flag;
}

// Thread per window: a window whose last cell continues starts a chain
// last -> mid* -> first, summed in position order.
__global__ void __launch_bounds__(kThreads) k_deposit_resolve(const uint32_t* __restrict__ skey, const StepState* __restrict__ st,
                                                              double* __restrict__ seg, uint32_t* __restrict__ stamp,
                                                              const double* __restrict__ carry_first,
                                                              const double* __restrict__ carry_last,
                                                              const int* __restrict__ wflag, long long nwin) {
    const long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (w >= nwin) return;
    if (!(wflag[w] & kWinLast)) return;
    const uint32_t key = skey[w * 32 + 31];
    double acc[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[c] = carry_last[(size_t)w * 8 + c];
    long long u = w + 1;
    while (u < nwin && (wflag[u] & kWinMid)) {
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[c] += carry_first[(size_t)u * 8 + c];
        ++u;
    }
    if (u < nwin && (wflag[u] & kWinFirst)) {
#pragma unroll
        for (int c = 0; c < 8; ++c) acc[c] += carry_first[(size_t)u * 8 + c];
    }
    double* s = seg + (size_t)key * 8;
#pragma unroll
    for (int c = 0; c < 8; ++c) s[c] = acc[c];
    stamp[key] = st->gen;
}

// rho(x,y,z) = (sum over the 8 cells touching the point of their corner sums)
// / dT * tmp2   (PartBunch.cpp:496, :510-511)
template <typename T>
__global__ void __launch_bounds__(kThreads) k_assemble_rho(BunchConst bc, const StepState* __restrict__ st,
                                                           const double* __restrict__ seg,
                                                           const uint32_t* __restrict__ stamp, T* __restrict__ rho) {
    const int n0 = bc.n[0], n1 = bc.n[1], n2 = bc.n[2];
    const long long M = (long long)n0 * n1 * n2;
    const unsigned gen = st->gen;
    const double dT = bc.dT, tmp2 = st->tmp2;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(c % n0);
        const int j = (int)((c / n0) % n1);
        const int k = (int)(c / ((long long)n0 * n1));
        double s = 0.0;
#pragma unroll
        for (int corner = 0; corner < 8; ++corner) {
            const int a = corner & 1, b = (corner >> 1) & 1, e = (corner >> 2) & 1;
            const int ci = i - a, cj = j - b, ck = k - e;
            if (ci < 0 || cj < 0 || ck < 0 || ci > n0 - 2 || cj > n1 - 2 || ck > n2 - 2) continue;
            const long long cell = ci + (long long)n0 * (cj + (long long)n1 * ck);
            if (stamp[cell] != gen) continue;
            s += seg[cell * 8 + corner];
        }
        s /= dT;
        s *= tmp2;
        rho[c] = (T)s;
    }
}

// ------------------------------------------------------------ Green's function
__device__ __forceinline__ double igf_antiderivative(double x, double y, double z, double cellVolume) {
    double r = sqrt(x * x + y * y + z * z);
    double tmpgrn = -z * z * atan(x * y / (z * r)) / 2;
    tmpgrn += -y * y * atan(x * z / (y * r)) / 2;
    tmpgrn += -x * x * atan(y * z / (x * r)) / 2;
    tmpgrn += y * z * log(x + r);
    tmpgrn += x * z * log(y + r);
    tmpgrn += x * y * log(z + r);
    return tmpgrn / cellVolume;
}

__global__ void __launch_bounds__(kThreads) k_igf_tmp(int n0, int n1, int n2, const StepState* __restrict__ st,
                                                      double* __restrict__ tmp) {
    const long long t0 = n0 + 2, t1 = n1 + 2, t2 = n2 + 2;
    const double h0 = st->hr_scaled[0], h1 = st->hr_scaled[1], h2 = st->hr_scaled[2];
    const double cellVolume = h0 * h1 * h2;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < t0 * t1 * t2; c += (long long)gridDim.x * blockDim.x) {
        const long long i = c % t0, j = (c / t0) % t1, k = c / (t0 * t1);
        const double vx = i * h0 - h0 / 2;
        const double vy = j * h1 - h1 / 2;
        const double vz = k * h2 - h2 / 2;
        tmp[c] = igf_antiderivative(vx, vy, vz, cellVolume);
    }
}

// G on (n0+1)(n1+1)(n2+1) points, 8-corner difference (:508-516), then
// G[0,0,0] <- G[0,0,1] (mirrorRhoField, :657).
__global__ void __launch_bounds__(kThreads) k_igf_G(int n0, int n1, int n2, const double* __restrict__ tmp,
                                                    double* __restrict__ G) {
    const long long g0 = n0 + 1, g1 = n1 + 1, g2 = n2 + 1;
    const long long t0 = n0 + 2, t1 = n1 + 2;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g0 * g1 * g2; c += (long long)gridDim.x * blockDim.x) {
        long long i = c % g0, j = (c / g0) % g1, k = c / (g0 * g1);
        if (c == 0) k = 1;
#define TG(a, b, e) tmp[(a) + t0 * ((b) + t1 * (e))]
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

// ------------------------------------------------------------ gradient
template <typename T>
__global__ void __launch_bounds__(kThreads) k_grad(BunchConst bc, const StepState* __restrict__ st, const T* __restrict__ phi,
                                                   T* __restrict__ E4) {
    const int n[3] = {bc.n[0], bc.n[1], bc.n[2]};
    const long long M = (long long)n[0] * n[1] * n[2];
    const long long stv[3] = {1, n[0], (long long)n[0] * n[1]};
    const double h[3] = {st->hr[0], st->hr[1], st->hr[2]};
    const double id[3] = {0.5 / h[0], 0.5 / h[1], 0.5 / h[2]};
    const double gz = st->gammaz;
    const double sc[3] = {gz / 1.0, gz / 1.0, 1.0 / (1.0 * gz)};
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < M; c += (long long)gridDim.x * blockDim.x) {
        const long long idx[3] = {c % n[0], (c / n[0]) % n[1], c / ((long long)n[0] * n[1])};
        double e[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const T* f = phi + c;
            const long long s = stv[d];
            double g;
            if (idx[d] == 0)
                g = id[d] * (-1.0 * (double)f[2 * s] + 4.0 * (double)f[s] - 3.0 * (double)f[0]);
            else if (idx[d] == n[d] - 1)
                g = id[d] * (1.0 * (double)f[-2 * s] - 4.0 * (double)f[-s] + 3.0 * (double)f[0]);
            else
                g = id[d] * ((double)f[s] - (double)f[-s]);
            e[d] = (-g) * sc[d];
        }
        E4[4 * c + 0] = (T)e[0];
        E4[4 * c + 1] = (T)e[1];
        E4[4 * c + 2] = (T)e[2];
        E4[4 * c + 3] = (T)0;
    }
}

// ------------------------------------------------------------ gather, kick, push
template <typename T>
__device__ __forceinline__ void cic_gather(const T* __restrict__ E4, const int* n, const int* l, const double* d, double* Ef) {
    const long long nx = n[0], nxy = (long long)n[0] * n[1];
    const long long b = l[0] + nx * l[1] + nxy * l[2];
    const long long o[8] = {b, b + 1, b + nx, b + nx + 1, b + nxy, b + nxy + 1, b + nxy + nx, b + nxy + nx + 1};
    const double w[8] = {(1 - d[0]) * (1 - d[1]) * (1 - d[2]), d[0] * (1 - d[1]) * (1 - d[2]),
                         (1 - d[0]) * d[1] * (1 - d[2]),       d[0] * d[1] * (1 - d[2]),
                         (1 - d[0]) * (1 - d[1]) * d[2],       d[0] * (1 - d[1]) * d[2],
                         (1 - d[0]) * d[1] * d[2],             d[0] * d[1] * d[2]};
    double e[8][3];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const T* p = E4 + 4 * o[k];
        e[k][0] = (double)p[0];
        e[k][1] = (double)p[1];
        e[k][2] = (double)p[2];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double s = w[0] * e[0][c];
#pragma unroll
        for (int k = 1; k < 8; ++k) s = s + w[k] * e[k][c];
        Ef[c] = s;
    }
}

template <typename T, bool STATS>
__global__ void __launch_bounds__(kThreads) k_gather_kick_push(BunchConst bc, double* __restrict__ x, double* __restrict__ y,
                                                               double* __restrict__ z, double* __restrict__ px,
                                                               double* __restrict__ py, double* __restrict__ pz,
                                                               const T* __restrict__ E4, StepState* st, double* partials,
                                                               unsigned* ticket) {
    __shared__ Trafo b2r, upd;
    __shared__ double hr[3], org[3], betaC;
    if (threadIdx.x == 0) {
        b2r = st->b2r;
        upd = st->upd;
        betaC = st->betaC;
        for (int k = 0; k < 3; ++k) {
            hr[k] = st->hr[k];
            org[k] = st->origin[k];
        }
    }
    __syncthreads();
    constexpr int NV = STATS ? 28 : 3;
    double acc[NV];
#pragma unroll
    for (int k = 0; k < NV; ++k) acc[k] = 0.0;
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        double X[3] = {x[i], y[i], z[i]};
        double P[3] = {px[i], py[i], pz[i]};
        int l[3];
        double d[3];
        if (!cic_locate(hr, org, bc.n, X, l, d)) bad = true;
        double Eb[3];
        cic_gather(E4, bc.n, l, d, Eb);
        double Bb[3] = {0.0 - betaC * Eb[1], 0.0 + betaC * Eb[0], 0.0};
        double R[3], Ef[3], Bf[3];
        trafo_transform_to(b2r, X, R);
        trafo_rotate_to(b2r, Eb, Ef);
        trafo_rotate_to(b2r, Bb, Bf);
        if (bc.bz_ext != 0.0) Bf[2] += bc.bz_ext;
        kick_one(P, Ef, Bf, bc.dT, bc.mass, bc.charge);
        push_one(R, P, bc.dT);
        double Ru[3], Pu[3];
        trafo_transform_to(upd, R, Ru);
        trafo_rotate_to(upd, P, Pu);
        x[i] = Ru[0];
        y[i] = Ru[1];
        z[i] = Ru[2];
        px[i] = Pu[0];
        py[i] = Pu[1];
        pz[i] = Pu[2];
        if constexpr (STATS) {
            accumulate_moments(acc, Ru, Pu);
        } else {
            acc[0] += Pu[0];
            acc[1] += Pu[1];
            acc[2] += Pu[2];
        }
    }
    if (bad) atomicOr(&st->err, kFlagGuard);
    block_sum<NV>(acc, partials);
    if (!last_block(ticket)) return;
    __shared__ double tot[NV];
    final_sum<NV>(partials, gridDim.x, tot);
    __syncthreads();
    if (threadIdx.x == 0) {
        StepState& s = *st;
        if constexpr (STATS) {
            for (int k = 0; k < 27; ++k) s.moments[k] = tot[k];
            s.gsum = tot[27];
            s.psum[0] = tot[1];
            s.psum[1] = tot[3];
            s.psum[2] = tot[5];
        } else {
            s.psum[0] = tot[0];
            s.psum[1] = tot[1];
            s.psum[2] = tot[2];
        }
        if (!derive_beam_frame(s, bc)) atomicOr(&s.err, kFlagFrame);
        s.step += 1;
        *ticket = 0u;
    }
}

// Fields only (PartBunch::computeSelfFields output): Ef, Bf in the beam frame,
// AoS (x, y, z per particle).
template <typename T>
__global__ void __launch_bounds__(kThreads) k_gather_fields(BunchConst bc, const double* __restrict__ x,
                                                            const double* __restrict__ y, const double* __restrict__ z,
                                                            const T* __restrict__ E4, StepState* st, double* __restrict__ Ef,
                                                            double* __restrict__ Bf) {
    const double hr[3] = {st->hr[0], st->hr[1], st->hr[2]};
    const double org[3] = {st->origin[0], st->origin[1], st->origin[2]};
    const double betaC = st->betaC;
    bool bad = false;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < bc.N; i += (long long)gridDim.x * blockDim.x) {
        double X[3] = {x[i], y[i], z[i]};
        int l[3];
        double d[3];
        if (!cic_locate(hr, org, bc.n, X, l, d)) bad = true;
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

}  // namespace

int particle_grid(const DevBunch& b) { return b.red_blocks; }

void launch_reduce_state(const DevBunch& b, bool init_frame, cudaStream_t s) {
    k_reduce_state<false><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.st, b.partials,
                                                           b.ticket, init_frame);
}

void launch_drift_to_beam(const DevBunch& b, bool drift, bool advance_ref, cudaStream_t s) {
    if (drift)
        k_drift_to_beam<true><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.st, b.partials,
                                                                b.ticket, advance_ref);
    else
        k_drift_to_beam<false><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz, b.st, b.partials,
                                                                 b.ticket, advance_ref);
}

void launch_cell_keys(const DevBunch& b, int digit_bits, cudaStream_t s) {
    const int te = sort_tile_elems();
    k_cell_keys<<<b.sort_tiles, kThreads, (1 << digit_bits) * sizeof(int), s>>>(b.bc, b.x, b.y, b.z, b.st, b.keys, b.hist,
                                                                               b.sort_tiles, te, digit_bits);
}

void launch_deposit(const DevBunch& b, cudaStream_t s) {
    const long long warps_per_block = kThreads / 32;
    const int g = (int)((b.nwin + warps_per_block - 1) / warps_per_block);
    k_deposit_windows<<<g, kThreads, 0, s>>>(b.bc, b.keys, b.vals, b.x, b.y, b.z, b.st, (double*)b.seg, b.stamp,
                                             (double*)b.carry_first, (double*)b.carry_last, b.wflag, b.nwin);
    const int g2 = (int)((b.nwin + kThreads - 1) / kThreads);
    k_deposit_resolve<<<g2, kThreads, 0, s>>>(b.keys, b.st, (double*)b.seg, b.stamp, (const double*)b.carry_first,
                                              (const double*)b.carry_last, b.wflag, b.nwin);
}

void launch_assemble_rho(const DevBunch& b, cudaStream_t s) {
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    const int g = grid_for(M, 148 * 16);
    if (b.precision == 0)
        k_assemble_rho<double><<<g, kThreads, 0, s>>>(b.bc, b.st, (const double*)b.seg, b.stamp, (double*)b.rho);
    else
        k_assemble_rho<float><<<g, kThreads, 0, s>>>(b.bc, b.st, (const double*)b.seg, b.stamp, (float*)b.rho);
}

void launch_igf(const DevBunch& b, const double* hr_host, cudaStream_t s) {
    (void)hr_host;
    const int n0 = b.bc.n[0], n1 = b.bc.n[1], n2 = b.bc.n[2];
    const long long T3 = (long long)(n0 + 2) * (n1 + 2) * (n2 + 2);
    const long long G3 = (long long)(n0 + 1) * (n1 + 1) * (n2 + 1);
    k_igf_tmp<<<grid_for(T3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.st, b.gtmp);
    k_igf_G<<<grid_for(G3, 148 * 16), kThreads, 0, s>>>(n0, n1, n2, b.gtmp, b.gline);
}

void launch_grad(const DevBunch& b, cudaStream_t s) {
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    const int g = grid_for(M, 148 * 16);
    if (b.precision == 0)
        k_grad<double><<<g, kThreads, 0, s>>>(b.bc, b.st, (const double*)b.phi, (double*)b.E4);
    else
        k_grad<float><<<g, kThreads, 0, s>>>(b.bc, b.st, (const float*)b.phi, (float*)b.E4);
}

void launch_gather_kick_push(const DevBunch& b, bool stats, cudaStream_t s) {
    if (b.precision == 0) {
        if (stats)
            k_gather_kick_push<double, true><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz,
                                                                              (const double*)b.E4, b.st, b.partials, b.ticket);
        else
            k_gather_kick_push<double, false><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz,
                                                                               (const double*)b.E4, b.st, b.partials, b.ticket);
    } else {
        if (stats)
            k_gather_kick_push<float, true><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz,
                                                                             (const float*)b.E4, b.st, b.partials, b.ticket);
        else
            k_gather_kick_push<float, false><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, b.px, b.py, b.pz,
                                                                              (const float*)b.E4, b.st, b.partials, b.ticket);
    }
}

void launch_gather_fields(const DevBunch& b, cudaStream_t s) {
    if (b.precision == 0)
        k_gather_fields<double><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, (const double*)b.E4, b.st, b.Ef, b.Bf);
    else
        k_gather_fields<float><<<b.red_blocks, kThreads, 0, s>>>(b.bc, b.x, b.y, b.z, (const float*)b.E4, b.st, b.Ef, b.Bf);
}

void launch_aos_to_soa(const double* aos, double* a, double* b, double* c, long long n, cudaStream_t s) {
    k_aos_to_soa<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(aos, a, b, c, n);
}

void launch_soa_to_aos(const double* a, const double* b, const double* c, double* aos, long long n, cudaStream_t s) {
    k_soa_to_aos<<<grid_for(n, 148 * 16), kThreads, 0, s>>>(a, b, c, aos, n);
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
