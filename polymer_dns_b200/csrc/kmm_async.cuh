// kmm_async.cuh -- mbarrier and one-dimensional bulk-copy helpers (sm_90+ PTX) for kernels that
// stage global rows into shared memory with the asynchronous copy engine.  Every wait is bounded:
// after the unit's limit (default 2 s) of %globaltimer it gives up and returns false, and the caller
// records an error.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace kasync {

__device__ __forceinline__ uint32_t sm_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(sm_addr(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the asynchronous proxy
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(sm_addr(bar)), "r"(bytes) : "memory");
}

// limit of the bounded waits in nanoseconds (default 2 s).  `static`: every translation unit that
// includes this header has its own copy, set through kasync_set_wait_limit from that unit.
static __device__ unsigned long long kasync_wait_ns = 2000000000ull;

// one test of phase `phase` of a barrier (the hardware may hold the thread for a while first)
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned phase) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(sm_addr(bar)), "r"(phase)
        : "memory");
    return done != 0;
}

// wait for phase `phase` of a barrier, at most `limit_ns` of %globaltimer; false if the limit ran
// out.  The first test comes before the timer is read, so a barrier that has already completed
// costs one instruction.
__device__ __forceinline__ bool mbar_wait_for(uint64_t *bar, unsigned phase, unsigned long long limit_ns) {
    if (mbar_try(bar, phase)) return true;
    const unsigned long long t0 = gtimer();
    for (;;) {
        if (mbar_try(bar, phase)) return true;
        if (gtimer() - t0 > limit_ns) return false;
    }
}

// the same with the unit's current limit (kasync_wait_ns, read only when the first test fails)
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase) {
    if (mbar_try(bar, phase)) return true;
    return mbar_wait_for(bar, phase, kasync_wait_ns);
}

// set this translation unit's wait limit on the current device (synchronous; not during capture)
static inline cudaError_t kasync_set_wait_limit(unsigned long long ns) {
    return cudaMemcpyToSymbol(kasync_wait_ns, &ns, sizeof(ns));
}

// global -> shared copy of `bytes` bytes (both addresses 16-byte aligned, bytes a multiple of 16),
// completing on `bar` (no multicast)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     sm_addr(dst)),
                 "l"(src), "r"(bytes), "r"(sm_addr(bar))
                 : "memory");
}

}  // namespace kasync
