// One-dimensional bulk copies (the Blackwell copy engine, cp.async.bulk) from global to
// shared memory, completing on a shared-memory mbarrier.  Used by the lexicographic tile
// kernel to stage each arc's parent run.  Rules the callers keep: source and destination
// 16-byte aligned, sizes multiples of 16 bytes, the total of one barrier phase below
// 2^20 bytes; no multicast; every wait bounded.
#pragma once

#include <cstdint>

namespace pmdd {
namespace dev {

__device__ __forceinline__ unsigned smem_addr(const void *p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// One thread; then a block barrier before any thread uses the mbarrier.
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrives once and announces `bytes` of bulk copies for the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// True once the phase of the given parity has completed (may suspend briefly).
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Orders this thread's earlier generic-proxy accesses to shared memory before later
// bulk-copy (async-proxy) writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// bytes (multiple of 16) from global src to shared dst (both 16-byte aligned).
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

}  // namespace dev
}  // namespace pmdd
