// fsg_mbar.cuh -- mbarrier waits with a bound, and bulk (TMA) global->shared copies.
#pragma once
#include <cstdint>

// Bound on an mbarrier wait: one second of %globaltimer (a chunk's copy completes in microseconds),
// and at most WAIT_POLLS polls whatever the timer reads
#define WAIT_NS 1000000000ull
#define WAIT_POLLS (1u << 26)

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 :: "r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}
// bounded wait for the phase with the given parity; false when the bound (bound_ns of %globaltimer, or
// WAIT_POLLS polls) was reached
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, unsigned long long bound_ns = WAIT_NS) {
    const unsigned a = smem_u32(bar);
    uint64_t start = 0;
    for (unsigned it = 0; it < WAIT_POLLS; it++) {
        unsigned done;
        asm volatile("{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
                     : "=r"(done) : "r"(a), "r"(parity) : "memory");
        if (done) return true;
        if ((it & 255u) == 0) {
            uint64_t now = global_ns();
            if (it == 0) start = now;
            else if (now - start > bound_ns) return false;
        }
    }
    return false;
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}
