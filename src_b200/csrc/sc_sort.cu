// sc_sort.cu -- counting sort of the particles by CIC cell.
//
// Cell keys are bounded by the mesh (key < n0 n1 n2), so one counting pass
// sorts them:
//   k_cell_keys (sc_particles.cu)  key and rank = atomicAdd(count[key], 1)
//   exclusive scan of count         -> first sorted position of every cell
//   k_scatter                       sorted key and particle index at start + rank
// The order of particles inside a cell depends on the order the atomics were
// served in; the deposit therefore sums each cell exactly (fixed point), so
// its result does not depend on that order and every run is bitwise the same.
#include "sc_internal.h"

namespace sc {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 16;
constexpr int kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int* total) {
    __shared__ int ws[kScanThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        int t = __shfl_up_sync(kFull, x, off);
        if (lane >= off) x += t;
    }
    if (lane == 31) ws[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int y = lane < (int)(blockDim.x >> 5) ? ws[lane] : 0;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            int t = __shfl_up_sync(kFull, y, off);
            if (lane >= off) y += t;
        }
        ws[lane] = y;
    }
    __syncthreads();
    const int before = (warp > 0 ? ws[warp - 1] : 0) + x - v;
    if (total) *total = ws[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

// out[i] = sum of in[0..i) (+ chunk_base[chunk]); chunk_sum[chunk] = chunk total
__global__ void __launch_bounds__(kScanThreads) k_scan_chunks(const int* __restrict__ in, int* __restrict__ out, long long n,
                                                              const int* __restrict__ chunk_base, int* __restrict__ chunk_sum) {
    const long long base = (long long)blockIdx.x * kScanChunk + (long long)threadIdx.x * kScanItems;
    int v[kScanItems];
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int run = block_exclusive_scan(s, &total);
    if (chunk_base) run += chunk_base[blockIdx.x];
    if (out) {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            if (base + k < n) out[base + k] = run;
            run += v[k];
        }
    }
    if (chunk_sum && threadIdx.x == 0) chunk_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(256) k_scatter(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ ranks,
                                                 const int* __restrict__ start, uint32_t* __restrict__ skey,
                                                 uint32_t* __restrict__ sval, long long n, int* __restrict__ err) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        const long long p = (long long)start[k] + ranks[i];
        if (p >= 0 && p < n) {
            skey[p] = k;
            sval[p] = (uint32_t)i;
        } else {
            atomicOr(err, kFlagSort);
        }
    }
}

}  // namespace

long long scan_scratch_ints(long long n) { return 2 * ((n + kScanChunk - 1) / kScanChunk) + 2; }

void exclusive_scan(const int* in, int* out, long long n, int* blocks, cudaStream_t s) {
    const long long chunks = (n + kScanChunk - 1) / kScanChunk;
    if (chunks <= 1) {
        k_scan_chunks<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, nullptr);
        return;
    }
    // chunk sums, scan of the sums (one chunk holds them for n <= 2^28), final pass
    k_scan_chunks<<<(unsigned)chunks, kScanThreads, 0, s>>>(in, nullptr, n, nullptr, blocks);
    k_scan_chunks<<<1, kScanThreads, 0, s>>>(blocks, blocks + chunks, chunks, nullptr, nullptr);
    k_scan_chunks<<<(unsigned)chunks, kScanThreads, 0, s>>>(in, out, n, blocks + chunks, nullptr);
}

// After k_cell_keys: b.keys (key per particle), b.vals_alt (rank in its
// cell), b.hist (count per cell).  Produces b.keys_alt (sorted keys) and
// b.vals (particle index per sorted position); b.hist_scan holds the cell starts.
void launch_sort(const DevBunch& b, cudaStream_t s) {
    const long long M = (long long)b.bc.n[0] * b.bc.n[1] * b.bc.n[2];
    exclusive_scan(b.hist, b.hist_scan, M, b.scan_blocks, s);
    long long g = (b.bc.N + 255) / 256;
    if (g > 148 * 16) g = 148 * 16;
    k_scatter<<<(unsigned)g, 256, 0, s>>>(b.keys, b.vals_alt, b.hist_scan, b.keys_alt, b.vals, b.bc.N, &b.st->err);
}

}  // namespace sc
