// sc_bulk.cuh -- bulk asynchronous copies global -> shared memory (the 1-D
// form of the Tensor Memory Accelerator, cp.async.bulk) completed on a
// shared-memory mbarrier, with bounded waits.
//
// A copy must start at 16-byte aligned global and shared addresses and move
// a multiple of 16 bytes; callers copy the 16-byte aligned body of a range
// and load a ragged tail element with a plain load.  No cluster multicast:
// every copy reads this GPU's own memory into the issuing block.
#pragma once

#include <cstdint>

namespace sc {

// wait iterations before a copy is declared lost (each try_wait itself
// suspends for a hardware-defined interval): far beyond any real copy
constexpr unsigned long long kBulkWaitIters = 1ull << 22;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes initialised barriers visible to the asynchronous (copy) proxy
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }

// one arrival that also announces `bytes` of copies completing on the barrier
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    uint64_t state;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;\n"
                 : "=l"(state)
                 : "r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    (void)state;
}

// global -> shared bulk copy of `bytes` (multiple of 16, both ends 16-byte aligned)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// true once the barrier's phase of parity `parity` has completed; false
// after kBulkWaitIters attempts
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    for (unsigned long long k = 0; k < kBulkWaitIters; ++k) {
        unsigned done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Stages element range [first, first + count) of up to three double arrays
// into shared memory: thread 0 issues the copies of the 16-byte aligned body
// (an even number of elements when `first` is even) and arms the barrier;
// the last element of an odd count is not copied (callers load it from
// global memory).  Returns the number of elements staged.
template <int NA>
__device__ __forceinline__ long long stage_doubles(double* const (&dst)[NA], const double* const (&src)[NA],
                                                   long long first, long long count, uint64_t* bar) {
    const long long body = count & ~1ll;
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(bar, (unsigned)(NA * body * sizeof(double)));
        if (body > 0)
#pragma unroll
            for (int a = 0; a < NA; ++a) bulk_g2s(dst[a], src[a] + first, (unsigned)(body * sizeof(double)), bar);
    }
    return body;
}

}  // namespace sc
