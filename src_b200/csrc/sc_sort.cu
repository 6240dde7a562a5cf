// sc_sort.cu -- stable LSD radix sort of the particles' cell keys.
//
// The deposit sums the particles of one cell in the order the sort leaves
// them; a stable sort whose first pass ranks particles by their index makes
// that order (cell, particle index) -- unique, so the deposit is bitwise
// reproducible.  Keys have at most 21 significant bits (128^3 cells); each
// pass sorts one digit of up to 9 bits.
//
//   upsweep    per-tile digit histogram, digit-major table [bins][tiles]
//   scan       exclusive prefix sum of that table (its flattened order is
//              exactly "all smaller digits, then earlier tiles")
//   downsweep  stable ranking inside the tile with warp match masks, scatter
#include "sc_internal.h"

namespace sc {
namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kItems = 16;
constexpr int kTile = kThreads * kItems;  // 4096 keys per tile
constexpr int kMaxBins = 512;
constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 8;
constexpr int kScanChunk = kScanThreads * kScanItems;

__global__ void __launch_bounds__(kThreads) k_upsweep(const uint32_t* __restrict__ keys, long long n, int shift, int bits,
                                                      int* __restrict__ hist, int tiles) {
    __shared__ int h[kMaxBins];
    const int bins = 1 << bits;
    for (int d = threadIdx.x; d < bins; d += blockDim.x) h[d] = 0;
    __syncthreads();
    const long long begin = (long long)blockIdx.x * kTile;
    long long end = begin + kTile;
    if (end > n) end = n;
    for (long long i = begin + threadIdx.x; i < end; i += blockDim.x) atomicAdd(&h[(keys[i] >> shift) & (bins - 1)], 1);
    __syncthreads();
    for (int d = threadIdx.x; d < bins; d += blockDim.x) hist[(size_t)d * tiles + blockIdx.x] = h[d];
}

// ---- exclusive scan of an int array (three phases for large arrays)
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

void exclusive_scan(const int* in, int* out, long long n, int* blocks, cudaStream_t s) {
    const long long chunks = (n + kScanChunk - 1) / kScanChunk;
    if (chunks <= 1) {
        k_scan_chunks<<<1, kScanThreads, 0, s>>>(in, out, n, nullptr, nullptr);
        return;
    }
    // chunk sums, scan of the sums (fits one chunk for n <= 64M), final pass
    k_scan_chunks<<<(unsigned)chunks, kScanThreads, 0, s>>>(in, nullptr, n, nullptr, blocks);
    k_scan_chunks<<<1, kScanThreads, 0, s>>>(blocks, blocks + chunks, chunks, nullptr, nullptr);
    k_scan_chunks<<<(unsigned)chunks, kScanThreads, 0, s>>>(in, out, n, blocks + chunks, nullptr);
}

// ---- downsweep: stable scatter of (key, value)
template <bool FIRST>
__global__ void __launch_bounds__(kThreads) k_downsweep(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin,
                                                        uint32_t* __restrict__ kout, uint32_t* __restrict__ vout, long long n,
                                                        int shift, int bits, const int* __restrict__ offsets, int tiles,
                                                        int* __restrict__ err) {
    __shared__ int cnt[kWarps][kMaxBins];
    __shared__ int run[kMaxBins];
    __shared__ int base[kMaxBins];
    const int bins = 1 << bits;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < bins; d += blockDim.x) {
        run[d] = 0;
        base[d] = offsets[(size_t)d * tiles + blockIdx.x];
    }
    const long long tile0 = (long long)blockIdx.x * kTile;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < kItems; ++r) {
        for (int e = threadIdx.x; e < kWarps * bins; e += blockDim.x) cnt[e / bins][e % bins] = 0;
        __syncthreads();
        const long long i = tile0 + (long long)r * kThreads + threadIdx.x;
        const bool valid = i < n;
        uint32_t key = 0, val = 0;
        int digit = bins;  // invalid lanes form their own group
        if (valid) {
            key = kin[i];
            val = FIRST ? (uint32_t)i : vin[i];
            digit = (int)((key >> shift) & (uint32_t)(bins - 1));
        }
        const unsigned peers = __match_any_sync(kFull, digit);
        const int lrank = __popc(peers & lt_mask);
        if (valid && lrank == 0) cnt[warp][digit] = __popc(peers);
        __syncthreads();
        // exclusive prefix over warps for each digit, continuing the tile's running count
        for (int d = threadIdx.x; d < bins; d += blockDim.x) {
            int acc = run[d];
            for (int w = 0; w < kWarps; ++w) {
                const int c = cnt[w][d];
                cnt[w][d] = acc;
                acc += c;
            }
            run[d] = acc;
        }
        __syncthreads();
        if (valid) {
            const long long p = (long long)base[digit] + cnt[warp][digit] + lrank;
            if (p >= 0 && p < n) {
                kout[p] = key;
                vout[p] = val;
            } else {
                atomicOr(err, kFlagSort);
            }
        }
        __syncthreads();
    }
}

}  // namespace

int sort_tile_elems() { return kTile; }

// Sorts b.keys (particle order) into b.keys / b.vals (cell order, values =
// particle indices).  The first pass's histogram comes from k_cell_keys.
void launch_sort(const DevBunch& b, cudaStream_t s) {
    const long long n = b.bc.N;
    const int bits_total = b.bc.key_bits;
    const int passes = (bits_total + 8) / 9;
    const int bits = (bits_total + passes - 1) / passes;
    const int tiles = b.sort_tiles;
    const long long table = (long long)tiles << bits;
    uint32_t* kin = b.keys;
    uint32_t* vin = b.vals;
    uint32_t* kout = b.keys_alt;
    uint32_t* vout = b.vals_alt;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * bits;
        if (p > 0) k_upsweep<<<tiles, kThreads, 0, s>>>(kin, n, shift, bits, b.hist, tiles);
        exclusive_scan(b.hist, b.hist_scan, table, b.scan_blocks, s);
        if (p == 0)
            k_downsweep<true><<<tiles, kThreads, 0, s>>>(kin, nullptr, kout, vout, n, shift, bits, b.hist_scan, tiles,
                                                          &b.st->err);
        else
            k_downsweep<false><<<tiles, kThreads, 0, s>>>(kin, vin, kout, vout, n, shift, bits, b.hist_scan, tiles,
                                                           &b.st->err);
        uint32_t* t = kin;
        kin = kout;
        kout = t;
        t = vin;
        vin = vout;
        vout = t;
    }
    // result must end in keys/vals
    if (kin != b.keys) {
        cudaMemcpyAsync(b.keys, kin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        cudaMemcpyAsync(b.vals, vin, n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
    }
}

int sort_digit_bits(int key_bits) {
    const int passes = (key_bits + 8) / 9;
    return (key_bits + passes - 1) / passes;
}

}  // namespace sc
