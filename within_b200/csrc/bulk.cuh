// bulk.cuh -- one-dimensional bulk copies global -> shared through the TMA
// engine (cp.async.bulk, no tensor map, no multicast) completing on a
// shared-memory mbarrier, and bounded waits on that barrier.
//
// A copy needs 16-byte aligned source and destination and a size that is a
// multiple of 16 bytes.  Every wait is bounded by the global timer: a wait
// that has not seen its phase complete after WAIT_LIMIT_NS returns false and
// the caller records an error and stops issuing.
#pragma once
#include <cstdint>

namespace wgpu {

constexpr unsigned long long WAIT_LIMIT_NS = 1000000000ull;   // 1 s
constexpr int ERR_WAIT_TIMEOUT = 9;                           // device error code of a timed-out wait

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes initialised barriers visible to the async proxy (the TMA engine)
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders earlier generic-proxy accesses of shared memory before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// one arrival that also announces `bytes` of transactions for the current phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of `parity` to complete; false after WAIT_LIMIT_NS.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (!mbar_test(bar, parity))
        if (global_ns() - t0 > WAIT_LIMIT_NS) return false;
    return true;
}

}  // namespace wgpu
