// mbar.cuh — mbarrier and bulk-copy (TMA) helpers shared by the kernels that stage data through shared memory with
// asynchronous bulk copies. Every wait is bounded (common.cuh).
#pragma once

#include "common.cuh"

namespace cspb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait for the phase of `parity`; false when the budget ran out or another thread gave up first.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, const volatile int* abort_flag,
                                          uint32_t* ctrl) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    for (;;) {
        if (mbar_test(bar, parity)) return true;
        if (*abort_flag || status_bad(ctrl)) return false;
        if (globaltimer_ns() - t0 > kWaitBudgetNs) {
            set_status(ctrl, CSPB_DEV_TIMEOUT);
            return false;
        }
    }
}
// One untiled bulk copy (TMA) of `bytes` from this GPU's global memory into this CTA's shared memory, completing on
// `bar`: both addresses 16-byte aligned, `bytes` a multiple of 16.
__device__ __forceinline__ void bulk_load_1d(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
// Bounded wait for the phase of `parity` that looks at nothing but the time: for a copy this thread's CTA has in
// flight, which must land before the CTA may leave even when another tile has given up. false after the budget.
__device__ __forceinline__ bool mbar_wait_own_copy(uint64_t* bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (!mbar_test(bar, parity))
        if (globaltimer_ns() - t0 > kWaitBudgetNs) return false;
    return true;
}
// Orders this thread's earlier generic-proxy accesses of shared memory before later async-proxy (TMA) ones.
__device__ __forceinline__ void fence_proxy_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

}  // namespace cspb

