// common.cuh — shared device helpers of libcspb: the workspace control block, bounded waits, a grid barrier.
//
// Every workspace starts with a 256-byte control block. Word 0 is the device status word (CSPB_DEV_* bits); the rest
// are counters the kernels use for dynamic work distribution and barriers. The host clears the block with one
// cudaMemsetAsync before each launch, so a call leaves nothing behind that the next one depends on.
//
// No device-side wait in this library can spin forever: each one polls %globaltimer and gives up after
// kWaitBudgetNs, sets CSPB_DEV_TIMEOUT in the status word and returns; every other waiter sees the status word and
// stops waiting too. The reference's ticket waits spin with no bound (cospanmdao/include/naga/cospan/kernel.hpp:215-236,
// examples/ns-residual/handwritten.hpp:71-79); these replace them.
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "../../include/cspb.h"

namespace cspb {

constexpr size_t kCtrlBytes = 256;  // the control block at the start of every workspace
constexpr unsigned long long kWaitBudgetNs = 2000000000ull;  // 2 s: every legitimate wait here ends in microseconds

// control-block word indices
enum CtrlWord : int {
    kStatus = 0,
    kBarrierCount = 1,
    kBarrierGen = 2,
    kWork0 = 4,  // dynamic work counters kWork0 .. kWork0 + 7
    kDone0 = 12, // completion counters kDone0 .. kDone0 + 7
    kDots0 = 32, // 4 f64 (words 32 .. 39): dot products one block forms for every block of the grid
};

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Programmatic dependent launch: a kernel started by cspb_host::launch_dependent() may run before the kernel ahead of
// it on the stream (cspb_host::clear_ctrl's) has finished; it calls pdl_wait() before its first access to what that
// kernel writes (the workspace's control block). Without such a launch it returns at once.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ uint64_t ld_acquire64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release64(uint64_t* p, uint64_t v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
// Single-copy-atomic 64-bit accesses at GPU scope, for words that carry a flag and a value together.
__device__ __forceinline__ uint64_t ld_relaxed64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed64(uint64_t* p, uint64_t v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_volatile(const uint32_t* p) {
    return *reinterpret_cast<const volatile uint32_t*>(p);
}

__device__ __forceinline__ void set_status(uint32_t* ctrl, uint32_t bits) { atomicOr(ctrl + kStatus, bits); }
__device__ __forceinline__ bool status_bad(const uint32_t* ctrl) { return ld_volatile(ctrl + kStatus) != 0u; }
// Only a wait that gave up (CSPB_DEV_TIMEOUT): for kernels whose data flags (a negative count, a total past 2^32 - 1)
// share the status word but must not end the other tiles' waits.
__device__ __forceinline__ bool status_timed_out(const uint32_t* ctrl) {
    return (ld_volatile(ctrl + kStatus) & CSPB_DEV_TIMEOUT) != 0u;
}

// Wait until *flag != old (acquire). Returns false (and sets CSPB_DEV_TIMEOUT) if the budget runs out or another
// waiter has already given up. Called by ONE thread.
__device__ __forceinline__ bool wait_change(const uint32_t* flag, uint32_t old, uint32_t* ctrl) {
    const unsigned long long t0 = globaltimer_ns();
    unsigned ns = 32;
    while (ld_acquire(flag) == old) {
        if (status_bad(ctrl)) return false;
        if (globaltimer_ns() - t0 > kWaitBudgetNs) {
            set_status(ctrl, CSPB_DEV_TIMEOUT);
            return false;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
    return true;
}

// Wait until *counter >= target (acquire). Same contract as wait_change.
__device__ __forceinline__ bool wait_at_least(const uint32_t* counter, uint32_t target, uint32_t* ctrl) {
    const unsigned long long t0 = globaltimer_ns();
    unsigned ns = 32;
    while (ld_acquire(counter) < target) {
        if (status_bad(ctrl)) return false;
        if (globaltimer_ns() - t0 > kWaitBudgetNs) {
            set_status(ctrl, CSPB_DEV_TIMEOUT);
            return false;
        }
        __nanosleep(ns);
        if (ns < 256) ns <<= 1;
    }
    return true;
}

// A sense-reversing grid barrier over gridDim.x blocks, all co-resident (the launches that use it are cooperative).
// Returns false for every block of the grid when the wait gave up, so callers return early together.
__device__ __forceinline__ bool grid_barrier(uint32_t* ctrl) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t* count = ctrl + kBarrierCount;
        uint32_t* gen = ctrl + kBarrierGen;
        const uint32_t g = ld_acquire(gen);
        __threadfence();
        const uint32_t arrived = atomicAdd(count, 1u);
        bool ok = true;
        if (arrived == gridDim.x - 1) {
            atomicExch(count, 0u);
            __threadfence();
            st_release(gen, g + 1u);
        } else {
            ok = wait_change(gen, g, ctrl);
        }
        s_ok = ok && !status_bad(ctrl);
    }
    __syncthreads();
    return s_ok != 0;
}

// One dynamic work item for the whole block from counter `word`.
__device__ __forceinline__ uint32_t grab_work(uint32_t* ctrl, int word, uint32_t amount = 1u) {
    __shared__ uint32_t s_item;
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(ctrl + word, amount);
    __syncthreads();
    return s_item;
}

// The next work item, fetched while the current one runs: thread 0 issues the atomic before the item's work and the
// block reads the value after it (the atomic's latency is hidden behind the item instead of preceding it).
__device__ __forceinline__ uint32_t prefetch_work(uint32_t* ctrl, int word, uint32_t amount = 1u) {
    return threadIdx.x == 0 ? atomicAdd(ctrl + word, amount) : 0u;
}
__device__ __forceinline__ uint32_t share_work(uint32_t v) {
    __shared__ uint32_t s_next;
    __syncthreads();
    if (threadIdx.x == 0) s_next = v;
    __syncthreads();
    return s_next;
}

// ---- loads and stores with cache hints -------------------------------------------------------------------------
// Streaming loads of data read once and never written by the kernel (evict-first in L2, no L1 allocation). Not
// volatile: the compiler may schedule them freely.
__device__ __forceinline__ uint64_t evict_first_policy() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ float4 ld_stream_f4(const float* p) {
    float4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "l"(p), "l"(evict_first_policy()));
    return v;
}
__device__ __forceinline__ uint4 ld_stream_u4(const void* p) {
    uint4 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
        : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
        : "l"(p), "l"(evict_first_policy()));
    return v;
}
__device__ __forceinline__ uint2 ld_stream_u2(const void* p) {
    uint2 v;
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v2.u32 {%0,%1}, [%2], %3;"
        : "=r"(v.x), "=r"(v.y)
        : "l"(p), "l"(evict_first_policy()));
    return v;
}
// Coherent loads through L2 (data written earlier in the same kernel by other blocks).
__device__ __forceinline__ float4 ld_cg_f4(const float* p) {
    float4 v;
    asm volatile("ld.global.cg.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p) : "memory");
    return v;
}
// Plain read-only loads (kept in L2 normally).
__device__ __forceinline__ float4 ld_nc_f4(const float* p) {
    float4 v;
    asm("ld.global.nc.v4.f32 {%0,%1,%2,%3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
    return v;
}
__device__ __forceinline__ void st_f4(float* p, float4 v) {
    asm volatile("st.global.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}
__device__ __forceinline__ void st_stream_f4(float* p, float4 v) {
    asm volatile("st.global.cs.v4.f32 [%0], {%1,%2,%3,%4};" ::"l"(p), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w) : "memory");
}

__device__ __forceinline__ float bf16_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

}  // namespace cspb

// ---- host side ---------------------------------------------------------------------------------------------------
namespace cspb_host {

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }
inline bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) % a) == 0; }

// The number of SMs and the cooperative-launch capability of the current device, cached per device.
struct DeviceInfo {
    int device = -1;
    int sms = 0;
    int coop = 0;
};
DeviceInfo device_info();

int map_cuda_error(cudaError_t e);

// Zeroes the control block at the start of a workspace (kCtrlBytes) with a one-block kernel that lets the next kernel
// on the stream start at once, if that kernel is launched with launch_dependent() (it must call pdl_wait() before it
// touches the control block). In place of cudaMemsetAsync: the separate operation and the gap after it cost about
// 2 µs before every launch, 3 % of a 4096² incompressible residual.
int clear_ctrl(void* ws, cudaStream_t st);
// A kernel launch allowed to start before the previous kernel on the stream has finished (programmatic stream
// serialization); a plain launch where the driver refuses it.
int launch_dependent(const void* kern, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void** args);

}  // namespace cspb_host
