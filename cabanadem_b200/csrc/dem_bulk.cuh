// dem_bulk.cuh -- bulk asynchronous copies (global -> shared) completed on an mbarrier, with
// bounded waits.  Used by the staged streaming kernel: one thread issues a tile's copies of
// contiguous SoA rows, the block waits on the tile's barrier phase.
//
// Every copy is the plain (non-tensor, non-multicast) cp.async.bulk from this GPU's global
// memory into the issuing CTA's shared memory: source and destination 16-byte aligned, the
// size a multiple of 16 bytes.
#pragma once
#include <cstdint>

namespace b200dem {
namespace bulk {

__device__ __forceinline__ uint32_t saddr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void bar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

// Makes initialised barriers visible to the copy engine (before the block barrier that
// publishes them).
__device__ __forceinline__ void bar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One arrival that also announces `bytes` of copies completing on this phase.
__device__ __forceinline__ void bar_arrive_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar))
        : "memory");
}

// L2 cache policy for data that every step reads again (the particle masses, contact words and
// neighbour lists between builds): its lines are evicted after the step's streaming data, so
// that they stay in L2 from one step to the next instead of coming from HBM each time.
__device__ __forceinline__ uint64_t policy_keep() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// copy_g2s with an L2 cache policy for the source lines.
__device__ __forceinline__ void copy_g2s_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                              uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(saddr(dst)),
        "l"(src), "r"(bytes), "r"(saddr(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ bool bar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase of the given parity; false after `limit` polls (each poll suspends the
// thread for a bounded, implementation-defined time), so a wait always ends.
__device__ __forceinline__ bool bar_wait(uint64_t *bar, uint32_t parity, int limit) {
    for (int k = 0; k < limit; ++k)
        if (bar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace bulk
}  // namespace b200dem
