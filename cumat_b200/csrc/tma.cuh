// Bulk-copy (TMA engine) and mbarrier helpers, inline PTX for sm_100a.
//
// Only the plain (non-multicast) forms are used: cp.async.bulk global ->
// shared memory of the issuing CTA, completion counted in bytes on an
// mbarrier. Every wait is bounded; a wait that runs out records an error code
// in a device word the host can read (cmcg_ctx_device_errors) and the caller
// skips the work instead of hanging.
#pragma once

#include <cstdint>

namespace cmcg {

constexpr uint32_t kWaitLimit = 1u << 24;   // try_wait rounds before giving up
enum : int32_t { DEVERR_MBAR_TIMEOUT = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes the initialised barriers visible to the async (bulk copy) proxy
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// bytes must be a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait (limit try_wait rounds) for the phase with the given parity;
// false if it timed out (the error is recorded in *err).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int32_t* err, uint32_t limit = kWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicOr(err, DEVERR_MBAR_TIMEOUT);
    return false;
}

// orders this thread's earlier generic-proxy accesses of shared memory before
// later bulk copies into it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace cmcg
