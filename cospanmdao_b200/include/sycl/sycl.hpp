// sycl/sycl.hpp — the subset of SYCL 2020 that CoSpan programs use, implemented on CUDA for sm_100a.
//
// This is not a SYCL implementation: it provides the names the cs:: API and the reference's example programs touch
// (ids and ranges, group functions inside a work-group, atomics, the math builtins, and an in-order queue with
// malloc / memset / memcpy / parallel_for) with CUDA underneath, so that their code compiles with nvcc and runs on
// the cspb runtime. A work-group is a CUDA block; group functions are block-wide; a queue is a CUDA stream.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#ifndef CS_HD
#define CS_HD __host__ __device__
#endif

namespace sycl {

// ---- ids and ranges -------------------------------------------------------------------------------------------
template <int R>
struct range {
    std::size_t v[R > 0 ? R : 1] = {};
    range() = default;
    template <class... I, class = std::enable_if_t<sizeof...(I) == R && (std::is_integral_v<I> && ...)>>
    CS_HD range(I... i) : v{static_cast<std::size_t>(i)...} {}
    CS_HD std::size_t& operator[](int d) { return v[d]; }
    CS_HD const std::size_t& operator[](int d) const { return v[d]; }
    CS_HD std::size_t get(int d) const { return v[d]; }
    CS_HD std::size_t size() const {
        std::size_t s = 1;
        for (int d = 0; d < R; ++d) s *= v[d];
        return s;
    }
    CS_HD friend bool operator==(const range& a, const range& b) {
        for (int d = 0; d < R; ++d)
            if (a.v[d] != b.v[d]) return false;
        return true;
    }
    CS_HD friend bool operator!=(const range& a, const range& b) { return !(a == b); }
};

template <int R>
struct id {
    std::size_t v[R > 0 ? R : 1] = {};
    id() = default;
    template <class... I, class = std::enable_if_t<sizeof...(I) == R && (std::is_integral_v<I> && ...)>>
    CS_HD id(I... i) : v{static_cast<std::size_t>(i)...} {}
    CS_HD std::size_t& operator[](int d) { return v[d]; }
    CS_HD const std::size_t& operator[](int d) const { return v[d]; }
    CS_HD std::size_t get(int d) const { return v[d]; }
    template <int Q = R, class = std::enable_if_t<Q == 1>>
    CS_HD operator std::size_t() const { return v[0]; }
};

template <int R>
struct nd_range {
    range<R> global, local;
    nd_range(range<R> g, range<R> l) : global(g), local(l) {}
    range<R> get_global_range() const { return global; }
    range<R> get_local_range() const { return local; }
};

// ---- functors -------------------------------------------------------------------------------------------------
template <class T = void>
struct plus {
    CS_HD T operator()(const T& a, const T& b) const { return a + b; }
};
template <class T = void>
struct minimum {
    CS_HD T operator()(const T& a, const T& b) const { return b < a ? b : a; }
};
template <class T = void>
struct maximum {
    CS_HD T operator()(const T& a, const T& b) const { return a < b ? b : a; }
};

// ---- math ---------------------------------------------------------------------------------------------------------
CS_HD inline float sqrt(float x) { return ::sqrtf(x); }
CS_HD inline double sqrt(double x) { return ::sqrt(x); }
CS_HD inline float sin(float x) { return ::sinf(x); }
CS_HD inline double sin(double x) { return ::sin(x); }
CS_HD inline float cos(float x) { return ::cosf(x); }
CS_HD inline double cos(double x) { return ::cos(x); }
CS_HD inline float fabs(float x) { return ::fabsf(x); }
CS_HD inline double fabs(double x) { return ::fabs(x); }
CS_HD inline float fmin(float a, float b) { return ::fminf(a, b); }
CS_HD inline float fmax(float a, float b) { return ::fmaxf(a, b); }

// ---- memory model -------------------------------------------------------------------------------------------------
enum class memory_order { relaxed, acquire, release, acq_rel, seq_cst };
enum class memory_scope { work_item, sub_group, work_group, device, system };
namespace access {
enum class address_space { global_space, local_space, generic_space, private_space };
enum class decorated { no, yes, legacy };
}  // namespace access

// Device intrinsics inside functions that component bodies call: those bodies are compiled for the host too (and
// never run there), so these functions are host-device with their device work under __CUDA_ARCH__.
#ifdef __CUDA_ARCH__
#define CS_DEV_ONLY(x) x
#else
#define CS_DEV_ONLY(x)
#endif

CS_HD inline void atomic_fence(memory_order, memory_scope s) {
    CS_DEV_ONLY(if (s == memory_scope::work_group) __threadfence_block(); else __threadfence();)
    (void)s;
}

// atomic_ref on global or shared memory (device scope). Floating-point min / max use compare-and-swap.
template <class T, memory_order O = memory_order::relaxed, memory_scope S = memory_scope::device,
          access::address_space A = access::address_space::generic_space>
class atomic_ref {
    T* p_;

public:
    CS_HD explicit atomic_ref(T& r) : p_(&r) {}
    CS_HD T load(memory_order o = O) const {
#ifdef __CUDA_ARCH__
        if (o == memory_order::relaxed) return *reinterpret_cast<volatile T*>(p_);
        T v = *reinterpret_cast<volatile T*>(p_);
        __threadfence();
        return v;
#else
        (void)o;
        return *p_;
#endif
    }
    CS_HD void store(T v, memory_order o = O) const {
#ifdef __CUDA_ARCH__
        if (o != memory_order::relaxed) __threadfence();
        *reinterpret_cast<volatile T*>(p_) = v;
#else
        (void)o;
        *p_ = v;
#endif
    }
    CS_HD T fetch_add(T v, memory_order = O) const {
#ifdef __CUDA_ARCH__
        return atomicAdd(p_, v);
#else
        const T old = *p_;
        *p_ = old + v;
        return old;
#endif
    }
    CS_HD T fetch_or(T v, memory_order = O) const {
#ifdef __CUDA_ARCH__
        return atomicOr(p_, v);
#else
        const T old = *p_;
        *p_ = old | v;
        return old;
#endif
    }
    CS_HD T exchange(T v, memory_order = O) const {
#ifdef __CUDA_ARCH__
        return atomicExch(p_, v);
#else
        const T old = *p_;
        *p_ = v;
        return old;
#endif
    }
    CS_HD T fetch_min(T v, memory_order = O) const {
#ifdef __CUDA_ARCH__
        if constexpr (std::is_floating_point_v<T>) {
            static_assert(sizeof(T) == 4, "floating-point atomic min is provided for float");
            unsigned* a = reinterpret_cast<unsigned*>(p_);
            unsigned old = *reinterpret_cast<volatile unsigned*>(a);
            while (__uint_as_float(old) > v || (__uint_as_float(old) != __uint_as_float(old))) {
                const unsigned prev = atomicCAS(a, old, __float_as_uint(v));
                if (prev == old) break;
                old = prev;
            }
            return __uint_as_float(old);
        } else {
            return atomicMin(p_, v);
        }
#else
        const T old = *p_;
        if (v < old) *p_ = v;
        return old;
#endif
    }
    CS_HD T fetch_max(T v, memory_order = O) const {
#ifdef __CUDA_ARCH__
        if constexpr (std::is_floating_point_v<T>) {
            static_assert(sizeof(T) == 4, "floating-point atomic max is provided for float");
            unsigned* a = reinterpret_cast<unsigned*>(p_);
            unsigned old = *reinterpret_cast<volatile unsigned*>(a);
            while (__uint_as_float(old) < v || (__uint_as_float(old) != __uint_as_float(old))) {
                const unsigned prev = atomicCAS(a, old, __float_as_uint(v));
                if (prev == old) break;
                old = prev;
            }
            return __uint_as_float(old);
        } else {
            return atomicMax(p_, v);
        }
#else
        const T old = *p_;
        if (old < v) *p_ = v;
        return old;
#endif
    }
    CS_HD bool compare_exchange_strong(T& expected, T desired, memory_order = O) const {
#ifdef __CUDA_ARCH__
        const T prev = atomicCAS(p_, expected, desired);
#else
        const T prev = *p_;
        if (prev == expected) *p_ = desired;
#endif
        const bool ok = prev == expected;
        expected = prev;
        return ok;
    }
};

// ---- work-groups (a CUDA block) ---------------------------------------------------------------------------------
namespace detail {
// block-wide scratch for the group functions (32 warp partials of up to 8 bytes, plus a broadcast slot)
CS_HD inline unsigned char* group_scratch() {
#ifdef __CUDA_ARCH__
    __shared__ __align__(16) unsigned char s[33 * 8];
    return s;
#else
    return nullptr;
#endif
}
CS_HD inline unsigned thread_x() {
#ifdef __CUDA_ARCH__
    return threadIdx.x;
#else
    return 0;
#endif
}
CS_HD inline unsigned block_x() {
#ifdef __CUDA_ARCH__
    return blockDim.x;
#else
    return 1;
#endif
}
CS_HD inline void sync_block() { CS_DEV_ONLY(__syncthreads();) }
template <class T>
CS_HD inline T shfl_xor(T x, int m) {
#ifdef __CUDA_ARCH__
    return __shfl_xor_sync(0xffffffffu, x, m);
#else
    (void)m;
    return x;
#endif
}
template <class T>
CS_HD inline T shfl_up(T x, int d) {
#ifdef __CUDA_ARCH__
    return __shfl_up_sync(0xffffffffu, x, d);
#else
    (void)d;
    return x;
#endif
}
}  // namespace detail

// The physical work-group of a launch: block-shaped, row-major (dimension D-1 fastest).
template <int D>
struct group {
    range<D> local;        // work-items per group
    range<D> grange;       // groups
    id<D> gid;             // this group
    CS_HD std::size_t get_local_linear_id() const { return detail::thread_x(); }
    CS_HD std::size_t get_local_linear_range() const { return detail::block_x(); }
    CS_HD range<D> get_local_range() const { return local; }
    CS_HD std::size_t get_local_range(int d) const { return local[d]; }
    CS_HD id<D> get_group_id() const { return gid; }
    CS_HD std::size_t get_group_id(int d) const { return gid[d]; }
    CS_HD range<D> get_group_range() const { return grange; }
    CS_HD std::size_t get_group_linear_id() const {
        std::size_t l = 0;
        for (int d = 0; d < D; ++d) l = l * grange[d] + gid[d];
        return l;
    }
};

template <int D>
CS_HD inline void group_barrier(const group<D>&, memory_scope = memory_scope::work_group) {
    detail::sync_block();
}

// A fixed-order block reduction: xor tree in each warp, then the warps in index order. Every work-item gets the result.
template <int D, class T, class Op>
CS_HD inline T reduce_over_group(const group<D>&, T x, Op op) {
    static_assert(sizeof(T) <= 8, "group reductions of values up to 8 bytes");
#ifdef __CUDA_ARCH__
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) x = op(x, __shfl_xor_sync(0xffffffffu, x, off));
    T* s = reinterpret_cast<T*>(detail::group_scratch());
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned warps = (blockDim.x + 31u) >> 5;
    __syncthreads();
    if (lane == 0) s[warp] = x;
    __syncthreads();
    T r = s[0];
    for (unsigned w = 1; w < warps; ++w) r = op(r, s[w]);
    __syncthreads();
    return r;
#else
    (void)op;
    return x;
#endif
}

template <int D, class T>
CS_HD inline T group_broadcast(const group<D>&, T x, std::size_t local_linear_id = 0) {
#ifdef __CUDA_ARCH__
    T* s = reinterpret_cast<T*>(detail::group_scratch() + 32 * 8);
    __syncthreads();
    if (threadIdx.x == local_linear_id) *s = x;
    __syncthreads();
    const T r = *s;
    __syncthreads();
    return r;
#else
    (void)local_linear_id;
    return x;
#endif
}

// inclusive / exclusive scans over a group (block): warp shuffles, then the warp offsets in order
template <int D, class T, class Op>
CS_HD inline T inclusive_scan_over_group(const group<D>&, T x, Op op) {
#ifdef __CUDA_ARCH__
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= unsigned(off)) x = op(x, o);
    }
    T* s = reinterpret_cast<T*>(detail::group_scratch());
    __syncthreads();
    if (lane == 31u || threadIdx.x == blockDim.x - 1) s[warp] = x;
    __syncthreads();
    T pre{};
    for (unsigned w = 0; w < warp; ++w) pre = w == 0 ? s[0] : op(pre, s[w]);
    __syncthreads();
    return warp == 0 ? x : op(pre, x);
#else
    (void)op;
    return x;
#endif
}
template <int D, class T, class Op>
CS_HD inline T exclusive_scan_over_group(const group<D>& g, T x, T init, Op op) {
#ifdef __CUDA_ARCH__
    const T inc = inclusive_scan_over_group(g, x, op);
    T* s = reinterpret_cast<T*>(detail::group_scratch() + 8);
    // the exclusive value of work-item t is the inclusive value of t - 1
    __syncthreads();
    T prev = __shfl_up_sync(0xffffffffu, inc, 1);
    if ((threadIdx.x & 31u) == 31u) s[threadIdx.x >> 5] = inc;
    __syncthreads();
    if ((threadIdx.x & 31u) == 0u && threadIdx.x != 0) prev = s[(threadIdx.x >> 5) - 1];
    __syncthreads();
    return threadIdx.x == 0 ? init : op(init, prev);
#else
    (void)g;
    (void)op;
    (void)x;
    return init;
#endif
}

// ---- nd_item (the physical item of a launch) --------------------------------------------------------------------
template <int D>
struct nd_item {
    group<D> g;
    CS_HD id<D> get_local_id() const {
        id<D> r;
        std::size_t l = detail::thread_x();
        for (int d = D - 1; d >= 0; --d) {
            r[d] = l % g.local[d];
            l /= g.local[d];
        }
        return r;
    }
    CS_HD std::size_t get_local_id(int d) const { return get_local_id()[d]; }
    CS_HD std::size_t get_local_linear_id() const { return detail::thread_x(); }
    CS_HD range<D> get_local_range() const { return g.local; }
    CS_HD std::size_t get_local_range(int d) const { return g.local[d]; }
    CS_HD group<D> get_group() const { return g; }
    CS_HD std::size_t get_group(int d) const { return g.gid[d]; }
    CS_HD range<D> get_group_range() const { return g.grange; }
    CS_HD std::size_t get_group_range(int d) const { return g.grange[d]; }
    CS_HD std::size_t get_group_linear_id() const { return g.get_group_linear_id(); }
    CS_HD std::size_t get_global_id(int d) const { return g.gid[d] * g.local[d] + get_local_id(d); }
    CS_HD id<D> get_global_id() const {
        id<D> r;
        const id<D> l = get_local_id();
        for (int d = 0; d < D; ++d) r[d] = g.gid[d] * g.local[d] + l[d];
        return r;
    }
    CS_HD range<D> get_global_range() const {
        range<D> r;
        for (int d = 0; d < D; ++d) r[d] = g.grange[d] * g.local[d];
        return r;
    }
};

// ---- host: devices, events, queues ---------------------------------------------------------------------------------
namespace info {
namespace device {
struct name {};
struct max_work_group_size {};
struct local_mem_size {};
}  // namespace device
}  // namespace info

class device {
    int ordinal_ = 0;

public:
    device() { cudaGetDevice(&ordinal_); }
    explicit device(int ordinal) : ordinal_(ordinal) {}
    template <class Sel>
    explicit device(const Sel&) { cudaGetDevice(&ordinal_); }
    int ordinal() const { return ordinal_; }
    template <class Info>
    auto get_info() const {
        cudaDeviceProp p{};
        cudaGetDeviceProperties(&p, ordinal_);
        if constexpr (std::is_same_v<Info, info::device::name>) return std::string(p.name);
        else if constexpr (std::is_same_v<Info, info::device::max_work_group_size>) return std::size_t(p.maxThreadsPerBlock);
        else return std::size_t(p.sharedMemPerBlockOptin);
    }
    friend bool operator==(const device& a, const device& b) { return a.ordinal_ == b.ordinal_; }
};
struct default_selector_t {};
inline constexpr default_selector_t default_selector_v{};

// An event: a CUDA event recorded on a stream (or a completed event when default-constructed).
class event {
    std::shared_ptr<CUevent_st> e_;

public:
    event() = default;
    explicit event(cudaStream_t s) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(e, s);
            e_.reset(e, [](cudaEvent_t x) { cudaEventDestroy(x); });
        }
    }
    cudaEvent_t native() const { return e_.get(); }
    void wait() const {
        if (e_) cudaEventSynchronize(e_.get());
    }
};

namespace property {
namespace queue {
struct in_order {};
}  // namespace queue
}  // namespace property
using async_handler = std::function<void()>;

template <class T, int D = 1>
class local_accessor;

namespace detail {
template <class F, int D>
__global__ void nd_kernel(F f, range<D> local, range<D> grange) {
    nd_item<D> it;
    it.g.local = local;
    it.g.grange = grange;
    std::size_t b = blockIdx.x;
    for (int d = D - 1; d >= 0; --d) {
        it.g.gid[d] = b % grange[d];
        b /= grange[d];
    }
    f(it);
}
template <class F, int D>
__global__ void range_kernel(F f, range<D> r, std::size_t total) {
    for (std::size_t t = std::size_t(blockIdx.x) * blockDim.x + threadIdx.x; t < total;
         t += std::size_t(gridDim.x) * blockDim.x) {
        id<D> i;
        std::size_t l = t;
        for (int d = D - 1; d >= 0; --d) {
            i[d] = l % r[d];
            l /= r[d];
        }
        f(i);
    }
}
template <class F>
__global__ void single_kernel(F f) { f(); }

inline void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string("sycl shim: ") + what + ": " + cudaGetErrorString(e));
}
}  // namespace detail

// The command group handler: records the dynamic local memory the kernel needs, then launches.
class handler {
public:
    explicit handler(cudaStream_t s) : s_(s) {}
    std::size_t reserve_local(std::size_t bytes, std::size_t align) {
        local_ = (local_ + align - 1) / align * align;
        const std::size_t off = local_;
        local_ += bytes;
        return off;
    }
    template <int D, class F>
    void parallel_for(nd_range<D> r, F f) {
        range<D> grange;
        for (int d = 0; d < D; ++d) grange[d] = r.global[d] / r.local[d];
        const std::size_t groups = grange.size(), threads = r.local.size();
        if (local_ > 48 * 1024)
            detail::check(cudaFuncSetAttribute(detail::nd_kernel<F, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(local_)), "local memory");
        detail::nd_kernel<F, D><<<unsigned(groups), unsigned(threads), local_, s_>>>(f, r.local, grange);
        detail::check(cudaGetLastError(), "parallel_for(nd_range)");
    }
    template <int D, class F>
    void parallel_for(range<D> r, F f) {
        const std::size_t total = r.size();
        if (total == 0) return;
        std::size_t blocks = (total + 255) / 256;
        if (blocks > 65535u * 16) blocks = 65535u * 16;
        detail::range_kernel<F, D><<<unsigned(blocks), 256, 0, s_>>>(f, r, total);
        detail::check(cudaGetLastError(), "parallel_for(range)");
    }
    template <class F>
    void single_task(F f) {
        detail::single_kernel<F><<<1, 1, 0, s_>>>(f);
        detail::check(cudaGetLastError(), "single_task");
    }
    void depends_on(const event& e) {
        if (e.native()) cudaStreamWaitEvent(s_, e.native(), 0);
    }
    void depends_on(const std::vector<event>& es) {
        for (const event& e : es) depends_on(e);
    }

private:
    cudaStream_t s_;
    std::size_t local_ = 0;
};

// Dynamic local memory: a slice of the launch's dynamic shared memory, reserved when the accessor is constructed.
template <class T, int D>
class local_accessor {
    std::size_t off_ = 0;

public:
    local_accessor() = default;
    local_accessor(range<D> r, handler& h) { off_ = h.reserve_local(r.size() * sizeof(T), alignof(T) < 16 ? 16 : alignof(T)); }
    CS_HD T* base() const {
#ifdef __CUDA_ARCH__
        extern __shared__ __align__(16) unsigned char sycl_dyn_local[];
        return reinterpret_cast<T*>(sycl_dyn_local + off_);
#else
        return nullptr;
#endif
    }
    CS_HD T& operator[](std::size_t i) const { return base()[i]; }
    struct multi_ptr {
        T* p;
        CS_HD T* get() const { return p; }
        CS_HD operator T*() const { return p; }
    };
    template <access::decorated Dd = access::decorated::no>
    CS_HD multi_ptr get_multi_ptr() const { return multi_ptr{base()}; }
    CS_HD T* get_pointer() const { return base(); }
};

// An in-order queue on its own CUDA stream.
class queue {
    std::shared_ptr<CUstream_st> s_;
    device dev_;

    void make() {
        cudaStream_t s = nullptr;
        detail::check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "queue");
        s_.reset(s, [](cudaStream_t x) { cudaStreamDestroy(x); });
    }

public:
    queue() { make(); }
    template <class... P>
    explicit queue(const device& d, P&&...) : dev_(d) {
        cudaSetDevice(d.ordinal());
        make();
    }
    cudaStream_t native() const { return s_.get(); }
    device get_device() const { return dev_; }
    template <class CGF>
    event submit(CGF&& cgf) {
        handler h(native());
        cgf(h);
        return event(native());
    }
    template <int D, class F>
    event parallel_for(range<D> r, F f) {
        handler h(native());
        h.parallel_for(r, f);
        return event(native());
    }
    template <int D, class F>
    event parallel_for(nd_range<D> r, F f) {
        handler h(native());
        h.parallel_for(r, f);
        return event(native());
    }
    template <class F>
    event single_task(F f) {
        handler h(native());
        h.single_task(f);
        return event(native());
    }
    event memset(void* p, int v, std::size_t bytes) {
        detail::check(cudaMemsetAsync(p, v, bytes, native()), "memset");
        return event(native());
    }
    event memcpy(void* dst, const void* src, std::size_t bytes) {
        detail::check(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, native()), "memcpy");
        return event(native());
    }
    void wait() { detail::check(cudaStreamSynchronize(native()), "wait"); }
    void wait_and_throw() { wait(); }
};

template <class T>
T* malloc_device(std::size_t count, const queue&) {
    void* p = nullptr;
    if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) return nullptr;
    return static_cast<T*>(p);
}
inline void free(void* p, const queue&) {
    if (p) cudaFree(p);
}

}  // namespace sycl
