// d4_bulk.cuh: shared-memory mbarriers and the untiled bulk copy (global ->
// shared, completing on an mbarrier), for producer/consumer pipelines inside
// one CTA.  No multicast: every copy lands in the issuing CTA's own shared
// memory.  Waits are bounded and report failure instead of spinning forever.
#pragma once
#include <cstdint>

namespace d4 {
namespace bulk {

constexpr long long kWaitLimit = 1ll << 22;  // polls (each with a short sleep): > 0.2 s

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Makes barrier initialisation visible to the async proxy (bulk copies).
__device__ __forceinline__ void fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the completion of the barrier's phase with `parity`.
__device__ __forceinline__ bool wait(uint64_t *bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (long long k = 0; k < kWaitLimit; ++k) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
        if (k > 64) __nanosleep(32);
    }
    return false;
}

// `bytes` (a multiple of 16) from global `src` to shared `dst` (both 16-byte
// aligned); completes `bytes` of the barrier's transaction count.
__device__ __forceinline__ void g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
        ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace bulk
}  // namespace d4
