// bph_bulk.h -- bulk (TMA, no multicast) copies from this GPU's global
// memory into shared memory, completed on mbarriers, with bounded waits:
// an expired wait sets kStatusTimeout in the caller's status word and the
// kernel runs on (its results are then reported invalid), so no CTA can
// hang on a copy.  Device code only; include after bph_internal.cuh.
#pragma once

#include <cstdint>

namespace bph {
namespace bulk {

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// One thread: order this CTA's earlier generic-proxy accesses of dst before
// the async-proxy write, then copy bytes (multiple of 16, both addresses
// 16-byte aligned) from global src to shared dst, completing on bar.
__device__ __forceinline__ void bulk_fill(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr int kWaitSpins = 1 << 20;  // try_wait rounds (each suspends at most a short hardware interval)

__device__ __forceinline__ void mbar_wait(uint64_t *bar, uint32_t parity, int *status) {
    for (int i = 0; i < kWaitSpins; ++i)
        if (mbar_try_wait(bar, parity)) return;
    atomicOr(status, kStatusTimeout);
}

// One thread: a copy completing on bar, without the expect_tx (another
// thread posts the expected bytes of the stage once).  Orders this thread's
// earlier generic-proxy accesses of the stage before the async-proxy write.
__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// The same with an L2 eviction policy (streams read once: evict_first).
__device__ __forceinline__ void bulk_copy_hint(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                               unsigned long long policy) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

// One arrival on bar that also expects `bytes` of copies in this phase.
__device__ __forceinline__ void mbar_expect(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

}  // namespace bulk
}  // namespace bph
