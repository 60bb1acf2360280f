// gpe_tma.cuh -- bulk asynchronous copies (TMA engine, cp.async.bulk, no
// tensor map, no multicast) and mbarrier helpers for staging pass tiles in
// shared memory.  Every wait is bounded by the global timer; on expiry the
// caller records GPE_ERR_TIMEOUT and returns.
#pragma once

#include <stdint.h>

namespace gpe {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// Order this CTA's generic-proxy shared-memory accesses before later
// async-proxy (bulk copy) accesses.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* m, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}

// Global -> shared bulk copy completing on mbarrier m.  dst, src 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(m))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t phase) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(m)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `phase` of m, at most limit_ns nanoseconds.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t phase, uint64_t limit_ns) {
    if (mbar_try_wait(m, phase)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(m, phase)) {
        if (global_ns() - t0 > limit_ns) return false;
    }
    return true;
}

}  // namespace gpe
