// bulk.cuh -- global -> shared bulk copies on the TMA engine (sm_90+ PTX
// `cp.async.bulk`, no tensor map) completed on an mbarrier.
//
// Rules the callers keep (the copy is not checked at run time):
//   - source and destination 16-byte aligned, size a multiple of 16 bytes;
//   - the source lies wholly inside one allocation (round the start down and
//     the end up to 16 bytes, with the array padded for the overhang);
//   - no multicast, and only this GPU's memory as the source.
// Every wait is bounded: past kBulkSpins polls it reports failure, and the
// caller records an error instead of reading the buffer.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace mb {

constexpr uint32_t kBulkSpins = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// One thread; then fence_barrier_init and a CTA barrier before first use.
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals) : "memory");
}

// One thread, after every thread is done with the barrier: the location may
// then be initialised again.
__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this CTA's earlier generic-proxy accesses to shared memory before
// the async-proxy writes of a bulk copy into the same buffer.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// The arrival of this phase, expecting `bytes` of copies to complete it.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Wait for the phase of parity `parity` to complete; false after `polls`
// polls (kBulkSpins by default).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t polls = kBulkSpins) {
    for (uint32_t i = 0; i < polls; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

}  // namespace mb
