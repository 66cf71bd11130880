// batched.cu — a ragged batch of independent GEMVERs in ONE persistent launch, with device-scanned offsets.
//
// The host passes only the sizes n[k] (on the device). The call then
//   1. k_plan: per instance, validates n, picks the tile geometry of its size bucket (from the tuning word), and
//      writes its sizes: matrix elements n·ld (ld = n rounded up to 8, so every row starts on 16 bytes for f32 and
//      bf16), vector elements n, f64 column partials strips·n, f32 row partials chunks·n, strip counters, units;
//   2. six decoupled-lookback scans (scan.cu) turn the sizes into u64 offsets — matrix and vector offsets go to the
//      caller's a_off / v_off (count + 1 entries; element offsets past 2^32 are the normal case: 4096 instances of
//      n ~ log-U[64, 4096] hold ≈ 8.4e9 elements);
//   3. k_run: a persistent grid pulls work items from one counter: first every pass-1 unit of every instance (read A,
//      write Â, f64 column partials), then every pass-2 unit (row dots with x). The block that finishes the last
//      pass-1 unit of a column chunk of an instance forms x over that chunk (strips in order) and publishes the
//      chunk's flag; a pass-2 unit waits (bounded) for the flag of its own chunk only, so x of a large instance is
//      formed by as many blocks as it has chunks, and pass 2 starts on a chunk as soon as that chunk is done. A
//      waiting block only ever waits on work that running blocks hold and that never waits itself, so the launch
//      needs no co-residency guarantee.
// Per-instance results do not depend on the rest of the batch: the geometry is a function of (n, dtype, tuning) and
// every reduction runs in a fixed order (rowpass.cuh).
#include "rowpass.cuh"

namespace cspb {
namespace batch {

constexpr int kThreads = kPassThreads;
// tuning word bits 8..9: consecutive work items a block takes at once (0: 4, 1: 1, 2: 2, 3: 8); bits 10..11: blocks
// per SM (0: as many as fit, 1: one fewer, 2: two, 3: one). Neither changes a result: every sum's order is fixed by
// (n, dtype, the bucket codes) alone.
__host__ __device__ inline uint32_t group_of(uint32_t tune) {
    const uint32_t c = (tune >> 8) & 3u;
    return c == 1 ? 1u : (c == 2 ? 2u : (c == 3 ? 8u : 4u));
}
__host__ __device__ inline int blocks_per_sm_of(uint32_t tune, int fit) {
    const uint32_t c = (tune >> 10) & 3u;
    const int b = c == 1 ? fit - 1 : (c == 2 ? 2 : (c == 3 ? 1 : fit));
    return b < 1 ? 1 : (b > fit ? fit : b);
}
constexpr int kSets = 7;  // a, v, p, w, s, u, c
enum { SA = 0, SV = 1, SP = 2, SW = 3, SS = 4, SU = 5, SC = 6 };

// tuning word: 2 bits per size bucket (n < 512, < 1024, < 2048, >= 2048): 0 -> WX 2, 1 -> WX 1, 2 -> WX 4
__host__ __device__ inline int bucket_of(uint32_t n) { return n < 512 ? 0 : (n < 1024 ? 1 : (n < 2048 ? 2 : 3)); }
__host__ __device__ inline int wx_of(uint32_t tune, uint32_t n) {
    const uint32_t c = (tune >> (2 * bucket_of(n))) & 3u;
    return c == 1 ? 1 : (c == 2 ? 4 : 2);
}
__host__ __device__ inline int rows_of(int wx) { return (8 / wx) * 32; }
__host__ __device__ inline int cols_of(int wx, bool bf16) { return wx * 32 * (bf16 ? 8 : 4); }

struct PlanK {
    int64_t count;
    const uint32_t* n;
    const cspb_gemver_task* tasks;  // task mode when not NULL
    uint32_t tune;
    int bf16;
    uint64_t* sizes;  // [kSets][count]
    uint8_t* wx;      // [count]
    uint32_t* ctrl;
};

__global__ void k_plan(PlanK g) {
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < g.count; k += int64_t(gridDim.x) * blockDim.x) {
        const int64_t n64 = g.tasks ? g.tasks[k].n : int64_t(g.n[k]);
        uint32_t n = (n64 >= 1 && n64 <= 65536) ? uint32_t(n64) : 0u;
        if (n == 0) {
            set_status(g.ctrl, CSPB_DEV_NEGATIVE);
            n = 0;
        }
        const int wx = wx_of(g.tune, n);
        const uint64_t ld = (uint64_t(n) + 7) / 8 * 8;
        const uint64_t S = rows_of(wx), CW = cols_of(wx, g.bf16 != 0);
        const uint64_t strips = (n + S - 1) / S, chunks = (n + CW - 1) / CW;
        g.wx[k] = uint8_t(wx);
        g.sizes[SA * g.count + k] = uint64_t(n) * ld;
        g.sizes[SV * g.count + k] = n;
        g.sizes[SP * g.count + k] = strips * n;
        g.sizes[SW * g.count + k] = chunks * n;
        g.sizes[SS * g.count + k] = strips;
        g.sizes[SU * g.count + k] = strips * chunks;
        g.sizes[SC * g.count + k] = chunks;
    }
}

struct RunK {
    int64_t count;
    const uint32_t* n;
    const cspb_gemver_task* tasks;  // task mode when not NULL
    const uint8_t* wx;
    const uint64_t* off[kSets];  // each count + 1
    uint64_t cap[SS + 1];        // capacities of a, v, p, w, s (elements)
    const void* A;
    const float *u1, *v1, *u2, *v2, *y, *z, *alpha, *beta;
    float *B, *x, *w;
    double* P;
    float* Wp;
    uint32_t* strip_done;
    uint32_t* chunk_done;  // [Σ units]: per instance, from its unit offset, one counter per column chunk
    uint32_t* x_ready;     // [Σ units]: likewise, one flag per column chunk
    uint64_t cap_units;
    uint32_t* ctrl;
    uint32_t group;  // work items per grab (group_of)
};

// the instance holding unit u (u_off[k] <= u < u_off[k+1]); instances with no units are skipped by construction
__device__ __forceinline__ int64_t find_instance(const uint64_t* uoff, int64_t count, uint64_t u) {
    int64_t lo = 0, hi = count;  // uoff[lo] <= u < uoff[hi]
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldcg(uoff + mid) <= u) lo = mid; else hi = mid;
    }
    return lo;
}

// The same, starting from the instance of the block's previous item: a block takes items in increasing order, so
// its next unit is usually in the same instance or a little later (two loads instead of a ~12-step search).
__device__ __forceinline__ int64_t find_instance_from(const uint64_t* uoff, int64_t count, uint64_t u, int64_t hint) {
    if (hint < 0 || hint >= count) return find_instance(uoff, count, u);
    const uint64_t a = __ldcg(uoff + hint), b = __ldcg(uoff + hint + 1);
    if (a <= u && u < b) return hint;
    if (a > u) return find_instance(uoff, count, u);
    int64_t lo = hint, hi = count;  // uoff[lo] <= u < uoff[hi] (uoff[count] is the total, > u)
    for (int64_t step = 1;; step <<= 1) {  // gallop forward to bracket u
        const int64_t t = lo + step;
        if (t >= count) break;
        if (__ldcg(uoff + t) > u) { hi = t; break; }
        lo = t;
    }
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (__ldcg(uoff + mid) <= u) lo = mid; else hi = mid;
    }
    return lo;
}

template <typename T>
__device__ __forceinline__ PassArgs instance_args(const RunK& g, int64_t k, int wx, bool bf16, bool& vec_ok,
                                                  const float*& z, float& beta, float*& x) {
    PassArgs a{};
    uint32_t n;
    if (g.tasks) {
        const cspb_gemver_task& t = g.tasks[k];
        n = uint32_t(t.n);
        a.src = t.A;
        a.lds = t.lda;
        a.dst = t.B;
        a.ldd = t.ldb;
        a.u1 = t.u1; a.v1 = t.v1; a.u2 = t.u2; a.v2 = t.v2;
        a.cyB = t.y;
        a.xv = t.x;
        a.rout1 = t.w;
        a.rscale1 = t.alpha;
        z = t.z;
        beta = t.beta;
        x = t.x;
        const int eb = bf16 ? 2 : 4;
        vec_ok = (reinterpret_cast<uintptr_t>(t.A) % 16 == 0) && ((t.lda * eb) % 16 == 0) &&
                 (t.B == nullptr || ((reinterpret_cast<uintptr_t>(t.B) % 16 == 0) && ((t.ldb * 4) % 16 == 0)));
    } else {
        n = g.n[k];
        const uint64_t ld = (uint64_t(n) + 7) / 8 * 8;
        const uint64_t ao = __ldcg(g.off[SA] + k), vo = __ldcg(g.off[SV] + k);
        a.src = static_cast<const T*>(g.A) + ao;
        a.lds = int64_t(ld);
        a.dst = g.B ? g.B + ao : nullptr;
        a.ldd = int64_t(ld);
        a.u1 = g.u1 + vo; a.v1 = g.v1 + vo; a.u2 = g.u2 + vo; a.v2 = g.v2 + vo;
        a.cyB = g.y + vo;
        a.xv = g.x + vo;
        a.rout1 = g.w + vo;
        a.rscale1 = g.alpha[k];
        z = g.z ? g.z + vo : nullptr;
        beta = g.beta[k];
        x = g.x + vo;
        vec_ok = true;  // rows padded to 8 elements, A and B 16-byte aligned (checked by the host)
    }
    a.n = n;
    a.rows = n;
    a.PB = g.P + __ldcg(g.off[SP] + k);
    a.Wp = g.Wp + __ldcg(g.off[SW] + k);
    a.strip_done = g.strip_done + __ldcg(g.off[SS] + k);
    const int64_t S = rows_of(wx), CW = cols_of(wx, bf16);
    a.strips = (n + S - 1) / S;
    a.chunks = (n + CW - 1) / CW;
    return a;
}

// x of one instance over columns [c0, c1) by one block: x[j] = z[j] + β · Σ_s P[s][j], strips in order (f64), then
// rounded.
__device__ __forceinline__ void instance_x(const PassArgs& a, const float* z, float beta, float* x, int64_t c0,
                                           int64_t c1) {
    for (int64_t j = c0 + threadIdx.x; j < c1; j += blockDim.x) {
        double s = 0.0;
        int64_t st = 0;
        for (; st + 8 <= a.strips; st += 8) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = __ldcg(a.PB + (st + k) * a.n + j);
#pragma unroll
            for (int k = 0; k < 8; ++k) s += v[k];
        }
        for (; st < a.strips; ++st) s += __ldcg(a.PB + st * a.n + j);
        const double zz = z ? double(__ldcg(z + j)) : 0.0;
        x[j] = float(zz + double(beta) * s);
    }
}

// x over [c0, c1) in the low-rank form (no Â): x[j] = z[j] + β · (Σ_s P[s][j] + v1[j]·s1 + v2[j]·s2), the strips in
// order as instance_x, s1 = u1·y and s2 = u2·y (block_dot2: every block of the instance forms the same two values).
__device__ __forceinline__ void instance_x_lr(const PassArgs& a, const float* z, float beta, float* x, int64_t c0,
                                              int64_t c1) {
    double s1, s2;
    block_dot2(a.u1, a.u2, a.cyB, a.n, s1, s2);
    for (int64_t j = c0 + threadIdx.x; j < c1; j += blockDim.x) {
        double s = 0.0;
        int64_t st = 0;
        for (; st + 8 <= a.strips; st += 8) {
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = __ldcg(a.PB + (st + k) * a.n + j);
#pragma unroll
            for (int k = 0; k < 8; ++k) s += v[k];
        }
        for (; st < a.strips; ++st) s += __ldcg(a.PB + st * a.n + j);
        s = __fma_rn(double(__ldcg(a.v1 + j)), s1, s);
        s = __fma_rn(double(__ldcg(a.v2 + j)), s2, s);
        const double zz = z ? double(__ldcg(z + j)) : 0.0;
        x[j] = float(zz + double(beta) * s);
    }
}

// rows in flight of the low-rank units (16-bit storage: 8, which keeps every variant of this kernel free of spills;
// the batching does not change the arithmetic)
template <typename T> inline constexpr int kLrRows = 8;

// Blocks per SM of a k_run variant: 3 for f32 and for the lean variant (80 registers, the instance's arguments in
// shared memory, 8-row load batches), 2 for the 16-bit variants that also form Â (128 registers).
template <typename T, bool LEAN> inline constexpr int kRunBlocks = (sizeof(T) == 4 || LEAN) ? 3 : 2;

// LR: an instance takes the low-rank form of cspb_gemver_fused with CSPB_GEMVER_LOWRANK: without Â, column sums of
// A·y, then row dots of A·x, the rank-2 terms in the finishes; with Â and a 16-bit A, pass 2 and the w finish only.
// LEAN: the variant for batches without Â (only the low-rank paths are compiled, so it fits 3 blocks per SM).
template <typename T, int WX, bool LR, bool LEAN>
__device__ __forceinline__ void unit1(const PassArgs& a, int64_t unit, bool vec_ok, unsigned char* smem) {
    if (LEAN || (LR && a.dst == nullptr)) pass_unit<T, WX, true, false, false, true, false, kLrRows<T>>(a, unit, vec_ok, smem);
    else pass_unit<T, WX, true, true, false, true, false, sizeof(T) == 4 ? 8 : 0>(a, unit, vec_ok, smem);
}
// Pass 2 reads the stored Â (f32) when there is one and the matrix is f32; otherwise A again, re-applying the update
// (or, low-rank, without it).
template <typename T, int WX, bool LR, bool LEAN>
__device__ __forceinline__ void unit2(const PassArgs& a, int64_t unit, bool vec_ok, unsigned char* smem) {
    if (LEAN) {  // no Â in the batch: a.dst is NULL
        pass_unit<T, WX, true, false, false, false, true, kLrRows<T>, true>(a, unit, vec_ok, smem);
    } else if (LR && (a.dst == nullptr || sizeof(T) == 2)) {  // low-rank: w from A (also when a 16-bit A's Â is stored)
        PassArgs b = a;
        b.dst = nullptr;  // pass 2 only reads A
        pass_unit<T, WX, true, false, false, false, true, kLrRows<T>, true>(b, unit, vec_ok, smem);
    } else if (sizeof(T) == 4 && a.dst != nullptr) {
        PassArgs b = a;
        b.src = a.dst;
        b.lds = a.ldd;
        b.dst = nullptr;  // pass 2 only reads Â
        pass_unit<float, WX, false, false, false, false, true, 8, true>(b, unit, vec_ok, smem);
    } else {
        pass_unit<T, WX, true, true, false, false, true, 0, true>(a, unit, vec_ok, smem);
    }
}

template <typename T, bool LR, bool LEAN = false>
__global__ void __launch_bounds__(kThreads, (kRunBlocks<T, LEAN>)) k_run(RunK g) {
    static_assert(!LEAN || LR, "the lean variant is the low-rank form");
    constexpr bool bf16 = sizeof(T) == 2;
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, 1>() > pass_smem_bytes<T, 4>()
                                                    ? pass_smem_bytes<T, 1>()
                                                    : pass_smem_bytes<T, 4>()];
    // the device-computed totals must fit the capacities the caller declared (decided by one thread, so the whole
    // block leaves together)
    const uint64_t U1 = __ldcg(g.off[SU] + g.count);
    __shared__ int s_go;
    if (threadIdx.x == 0) {
        // the work list (at most 4·U1 items) must fit the 32-bit counter with room for its overshoot
        bool fits = 4 * U1 < 0xffffffffull - (1ull << 24) && U1 <= g.cap_units;
        for (int s = 0; s <= SS; ++s)  // task mode has no packed matrix / vector offsets
            if (g.off[s] != nullptr) fits = fits && __ldcg(g.off[s] + g.count) <= g.cap[s];
        if (!fits) set_status(g.ctrl, CSPB_DEV_CAPACITY);
        s_go = fits && !status_bad(g.ctrl);  // status set by the plan: an invalid size
    }
    __syncthreads();
    if (!s_go) return;
    // The work list, one counter: [pass-1 units][x finishes, one per (instance, chunk)][pass-2 units]
    // [w finishes, one per (instance, strip)]. A unit only counts itself done (a release reduction, no wait); a
    // finish waits (bounded) for the counter it needs and then forms x over a chunk or w over a strip, in the fixed
    // orders of the single-instance kernels. Everything an item waits for sits earlier in the list, taken by blocks
    // that are running and never wait on later items.
    const uint64_t C1 = __ldcg(g.off[SC] + g.count), S1 = __ldcg(g.off[SS] + g.count);
    const uint64_t e1 = U1, e2 = U1 + C1, e3 = 2 * U1 + C1, e4 = 2 * U1 + C1 + S1;
    __shared__ int s_ok;
    int64_t cur = -1;
    // the instance's arguments: in shared memory for the 3-block variants, written by one thread per instance change,
    // so that they do not hold ~40 registers across the work loop; in registers otherwise
    constexpr bool kSharedArgs = kRunBlocks<T, LEAN> == 3;
    __shared__ PassArgs s_args;
    PassArgs a_reg{};
    PassArgs& a = kSharedArgs ? s_args : a_reg;
    bool vec_ok = false;
    const float* z = nullptr;
    float beta = 0.f;
    float* x = nullptr;
    int wx = 2;
    uint64_t ubase = 0, sbase = 0;
    auto instance = [&](int64_t k) {
        if (k == cur) return;
        cur = k;
        wx = g.wx[k];
        ubase = __ldcg(g.off[SU] + k);
        sbase = __ldcg(g.off[SS] + k);
        if constexpr (kSharedArgs) {  // called by the whole block between items (the previous one ended with a barrier)
            PassArgs t = instance_args<T>(g, k, wx, bf16, vec_ok, z, beta, x);
            if (threadIdx.x == 0) {
                if (LEAN && t.dst != nullptr) {  // a task with B under CSPB_BATCH_NO_B: the call fails, no B is written
                    set_status(g.ctrl, CSPB_DEV_ARGUMENT);
                    t.dst = nullptr;
                }
                s_args = t;
            }
            __syncthreads();
        } else {
            a = instance_args<T>(g, k, wx, bf16, vec_ok, z, beta, x);
        }
    };
    auto count_done = [&](uint32_t* counter) {  // this block's unit is complete
        __syncthreads();
        if (threadIdx.x == 0) asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(counter) : "memory");
    };
    auto wait_for = [&](const uint32_t* counter, uint32_t target) {  // bounded; false when it gave up
        if (threadIdx.x == 0) s_ok = ld_acquire(counter) >= target || wait_at_least(counter, target, g.ctrl);
        __syncthreads();
        return s_ok != 0;
    };
    const uint32_t group = g.group;
    for (uint32_t base = grab_work(g.ctrl, kWork0, group); uint64_t(base) < e4;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0, group);
        bool stop = false;
        for (uint32_t q = 0; q < group && !stop; ++q) {
            const uint64_t item = uint64_t(base) + q;
            if (item >= e4) break;
            if (item < e1 || (item >= e2 && item < e3)) {  // a unit of pass 1 or pass 2
                const bool pass2 = item >= e2;
                const uint64_t u = pass2 ? item - e2 : item;
                const int64_t k = find_instance_from(g.off[SU], g.count, u, cur);
                instance(k);
                const int64_t unit = int64_t(u - ubase);
                const int64_t c = unit % a.chunks, strip = unit / a.chunks;
                if (!pass2) {
                    switch (wx) {
                        case 1: unit1<T, 1, LR, LEAN>(a, unit, vec_ok, smem); break;
                        case 4: unit1<T, 4, LR, LEAN>(a, unit, vec_ok, smem); break;
                        default: unit1<T, 2, LR, LEAN>(a, unit, vec_ok, smem); break;
                    }
                    count_done(g.chunk_done + ubase + uint64_t(c));
                } else {
                    if (!wait_for(g.x_ready + ubase + uint64_t(c), 1u)) { stop = true; break; }
                    switch (wx) {
                        case 1: unit2<T, 1, LR, LEAN>(a, unit, vec_ok, smem); break;
                        case 4: unit2<T, 4, LR, LEAN>(a, unit, vec_ok, smem); break;
                        default: unit2<T, 2, LR, LEAN>(a, unit, vec_ok, smem); break;
                    }
                    count_done(g.strip_done + sbase + uint64_t(strip));
                }
            } else if (item < e2) {  // x over one chunk of an instance
                const uint64_t f = item - e1;
                const int64_t k = find_instance_from(g.off[SC], g.count, f, cur);
                instance(k);
                const int64_t c = int64_t(f - __ldcg(g.off[SC] + k));
                if (!wait_for(g.chunk_done + ubase + uint64_t(c), uint32_t(a.strips))) { stop = true; break; }
                const int64_t CW = cols_of(wx, bf16);
                const int64_t c1 = (c + 1) * CW < a.n ? (c + 1) * CW : a.n;
                if (LEAN || (LR && a.dst == nullptr)) instance_x_lr(a, z, beta, x, c * CW, c1);
                else instance_x(a, z, beta, x, c * CW, c1);
                __syncthreads();
                if (threadIdx.x == 0) {
                    __threadfence();
                    st_release(g.x_ready + ubase + uint64_t(c), 1u);
                }
            } else {  // w over one strip of an instance: the row-dot partials of its chunks, in chunk order
                const uint64_t f = item - e3;
                const int64_t k = find_instance_from(g.off[SS], g.count, f, cur);
                instance(k);
                const int64_t strip = int64_t(f - sbase);
                if (!wait_for(g.strip_done + sbase + uint64_t(strip), uint32_t(a.chunks))) { stop = true; break; }
                const int64_t S = rows_of(wx);
                const bool lr = LEAN || (LR && (a.dst == nullptr || bf16));  // as unit2
                double t1 = 0.0, t2 = 0.0;
                if (lr) block_dot2(a.v1, a.v2, a.xv, a.n, t1, t2);  // x is complete: every chunk fed this strip
                for (int64_t row = strip * S + threadIdx.x; row < (strip + 1) * S && row < a.n; row += blockDim.x) {
                    float sum = 0.f;
                    int64_t cc = 0;
                    for (; cc + 16 <= a.chunks; cc += 16) {
                        float v[16];
#pragma unroll
                        for (int t = 0; t < 16; ++t) v[t] = __ldcg(a.Wp + (cc + t) * a.n + row);
#pragma unroll
                        for (int t = 0; t < 16; ++t) sum += v[t];
                    }
                    for (; cc < a.chunks; ++cc) sum += __ldcg(a.Wp + cc * a.n + row);
                    if (lr) {
                        double dd = double(sum);
                        dd = __fma_rn(double(__ldcg(a.u1 + row)), t1, dd);
                        dd = __fma_rn(double(__ldcg(a.u2 + row)), t2, dd);
                        a.rout1[row] = float(double(a.rscale1) * dd);
                    } else {
                        a.rout1[row] = a.rscale1 * sum;
                    }
                }
            }
            __syncthreads();  // s_ok and the unit's shared memory are reused by the next item
        }
        if (stop) break;
        base = share_work(next);
    }
}

}  // namespace batch
}  // namespace cspb

using namespace cspb;
using cspb_host::align_up;
using cspb_host::aligned;

namespace {

struct BatchLayout {
    size_t off_sizes = 0, off_offs = 0, off_wx = 0, off_p1 = 0, off_xr = 0, off_scan = 0, off_P = 0, off_W = 0,
           off_S = 0, total = 0;
    uint64_t capP = 0, capW = 0, capS = 0, capU = 0;
};

BatchLayout batch_layout(int64_t count, int64_t max_elems, int64_t max_vec) {
    BatchLayout L;
    const uint64_t Smin = 64, CWmin = 128;  // the smallest strip and chunk of any tuning
    L.capP = uint64_t(max_elems) / Smin + uint64_t(max_vec);
    L.capW = uint64_t(max_elems) / CWmin + uint64_t(max_vec);
    L.capS = uint64_t(max_vec) / Smin + uint64_t(count);
    // units of an instance: ceil(n/S)·ceil(n/CW) <= n²/(S·CW) + n/S + n/CW + 1 <= n²/8192 + n/32 + 1
    L.capU = uint64_t(max_elems) / (Smin * CWmin) + uint64_t(max_vec) / 32 + uint64_t(count);
    size_t o = kCtrlBytes;
    L.off_sizes = o;
    o = align_up(o + size_t(batch::kSets) * size_t(count) * 8, 256);
    L.off_offs = o;  // p, w, s, u, c offsets (a and v go to the caller)
    o = align_up(o + 5 * size_t(count + 1) * 8, 256);
    L.off_wx = o;
    o = align_up(o + size_t(count), 256);
    L.off_p1 = o;  // chunk counters then chunk flags, zeroed together with the strip counters
    o = align_up(o + size_t(L.capU) * 4, 256);
    L.off_xr = o;
    o = align_up(o + size_t(L.capU) * 4, 256);
    L.off_S = o;
    o = align_up(o + size_t(L.capS) * 4, 256);
    L.off_scan = o;
    o = align_up(o + cspb_scan_workspace_bytes(count), 256);
    L.off_P = o;
    o = align_up(o + size_t(L.capP) * 8, 256);
    L.off_W = o;
    o = align_up(o + size_t(L.capW) * 4, 256);
    L.total = o;
    return L;
}

}  // namespace

extern "C" {

size_t cspb_gemver_batched_workspace_bytes(int64_t count, int64_t max_elems, int64_t max_vec) {
    if (count < 1 || max_elems < 1 || max_vec < 1) return 0;
    return batch_layout(count, max_elems, max_vec).total;
}

int cspb_gemver_batched_tunings(void) { return 1 << 12; }

}  // extern "C"

namespace {

// The plan, the six scans and the run, for the packed layout (tasks == NULL) or a task table.
int run_batch(int64_t count, int64_t max_elems, int64_t max_vec, int32_t a_dtype, int32_t tune, const uint32_t* n,
              const cspb_gemver_task* tasks, const cspb_gemver_batched_desc* d, uint64_t* a_off, uint64_t* v_off,
              void* workspace, size_t workspace_bytes, void* stream) {
    if (count < 1 || count > (int64_t(1) << 26) || max_elems < 1 || max_vec < 1) return CSPB_ERR_ARGUMENT;
    if (a_dtype != CSPB_F32 && a_dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    const bool lowrank = (tune & CSPB_BATCH_LOWRANK) != 0;
    const bool no_b = (tune & CSPB_BATCH_NO_B) != 0;
    tune &= ~(CSPB_BATCH_LOWRANK | CSPB_BATCH_NO_B);
    if (tune < 0 || tune >= cspb_gemver_batched_tunings()) return CSPB_ERR_UNSUPPORTED;
    for (uint32_t b = 0; b < 4; ++b)
        if (((uint32_t(tune) >> (2 * b)) & 3u) == 3u) return CSPB_ERR_UNSUPPORTED;
    const BatchLayout L = batch_layout(count, max_elems, max_vec);
    if (!workspace || !aligned(workspace, 256) || workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    const bool bf16 = a_dtype == CSPB_BF16;
    // control block, chunk counters and flags, strip counters: zeroed per call
    if (cudaMemsetAsync(ws, 0, kCtrlBytes, st) != cudaSuccess) return CSPB_ERR_CUDA;
    if (cudaMemsetAsync(ws + L.off_p1, 0, L.off_scan - L.off_p1, st) != cudaSuccess) return CSPB_ERR_CUDA;

    batch::PlanK pk{};
    pk.count = count;
    pk.n = n;
    pk.tasks = tasks;
    pk.tune = uint32_t(tune);
    pk.bf16 = bf16;
    pk.sizes = reinterpret_cast<uint64_t*>(ws + L.off_sizes);
    pk.wx = reinterpret_cast<uint8_t*>(ws + L.off_wx);
    pk.ctrl = reinterpret_cast<uint32_t*>(ws);
    int64_t pb = (count + 255) / 256;
    if (pb > 4096) pb = 4096;
    batch::k_plan<<<unsigned(pb), 256, 0, st>>>(pk);
    if (cudaGetLastError() != cudaSuccess) return CSPB_ERR_LAUNCH;

    uint64_t* offs = reinterpret_cast<uint64_t*>(ws + L.off_offs);
    uint64_t* outs[batch::kSets] = {a_off, v_off, offs, offs + (count + 1), offs + 2 * (count + 1),
                                    offs + 3 * (count + 1), offs + 4 * (count + 1)};
    for (int s = 0; s < batch::kSets; ++s) {
        if (!outs[s]) continue;  // task mode: no packed matrix / vector offsets
        const int r = cspb_exclusive_scan_u64(pk.sizes + size_t(s) * size_t(count), outs[s], count, ws + L.off_scan,
                                              cspb_scan_workspace_bytes(count), stream);
        if (r != CSPB_OK) return r;
    }

    batch::RunK g{};
    g.count = count;
    g.n = n;
    g.tasks = tasks;
    g.wx = pk.wx;
    for (int s = 0; s < batch::kSets; ++s) g.off[s] = outs[s];
    g.cap[batch::SA] = tasks ? ~0ull : uint64_t(max_elems);
    g.cap[batch::SV] = tasks ? ~0ull : uint64_t(max_vec);
    g.cap[batch::SP] = L.capP;
    g.cap[batch::SW] = L.capW;
    g.cap[batch::SS] = L.capS;
    if (d) {
        g.A = d->A;
        g.u1 = d->u1; g.v1 = d->v1; g.u2 = d->u2; g.v2 = d->v2; g.y = d->y; g.z = d->z;
        g.alpha = d->alpha;
        g.beta = d->beta;
        g.B = d->B;
        g.x = d->x;
        g.w = d->w;
    }
    g.P = reinterpret_cast<double*>(ws + L.off_P);
    g.Wp = reinterpret_cast<float*>(ws + L.off_W);
    g.strip_done = reinterpret_cast<uint32_t*>(ws + L.off_S);
    g.chunk_done = reinterpret_cast<uint32_t*>(ws + L.off_p1);
    g.x_ready = reinterpret_cast<uint32_t*>(ws + L.off_xr);
    g.cap_units = L.capU;
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    // without Â anywhere in the batch, a 16-bit low-rank batch runs the lean variant (3 blocks per SM)
    const bool lean = bf16 && lowrank && (d ? d->B == nullptr : no_b);
    const void* kern = lean ? reinterpret_cast<const void*>(batch::k_run<__nv_bfloat16, true, true>)
                     : bf16 ? (lowrank ? reinterpret_cast<const void*>(batch::k_run<__nv_bfloat16, true>)
                                       : reinterpret_cast<const void*>(batch::k_run<__nv_bfloat16, false>))
                            : (lowrank ? reinterpret_cast<const void*>(batch::k_run<float, true>)
                                       : reinterpret_cast<const void*>(batch::k_run<float, false>));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, batch::kThreads, 0) != cudaSuccess || per_sm < 1)
        return CSPB_ERR_LAUNCH;
    per_sm = batch::blocks_per_sm_of(uint32_t(tune), per_sm);
    g.group = batch::group_of(uint32_t(tune));
    void* args[] = {&g};
    if (cudaLaunchKernel(kern, dim3(unsigned(per_sm * di.sms)), dim3(batch::kThreads), args, 0, st) != cudaSuccess)
        return CSPB_ERR_LAUNCH;
    return CSPB_OK;
}

}  // namespace

extern "C" {

int cspb_gemver_batched(const cspb_gemver_batched_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (!d->n || !d->A || !d->u1 || !d->v1 || !d->u2 || !d->v2 || !d->y || !d->alpha || !d->beta || !d->x || !d->w ||
        !d->a_off || !d->v_off)
        return CSPB_ERR_ARGUMENT;
    if (!aligned(d->A, 16) || (d->B && !aligned(d->B, 16))) return CSPB_ERR_ARGUMENT;
    return run_batch(d->count, d->max_elems, d->max_vec, d->a_dtype, d->tune, d->n, nullptr, d, d->a_off, d->v_off,
                     d->workspace, d->workspace_bytes, stream);
}

int cspb_gemver_tasks(const cspb_gemver_task* tasks, int64_t count, int64_t max_elems, int64_t max_vec,
                      int32_t a_dtype, int32_t tune, void* workspace, size_t workspace_bytes, void* stream) {
    if (!tasks) return CSPB_ERR_ARGUMENT;
    return run_batch(count, max_elems, max_vec, a_dtype, tune, nullptr, tasks, nullptr, nullptr, nullptr, workspace,
                     workspace_bytes, stream);
}

}  // extern "C"
