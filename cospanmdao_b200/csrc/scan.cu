// scan.cu — single-pass exclusive scan (decoupled lookback) of u32 / u64, and the fused ragged-column builder.
//
// Replaces cs::detail::exclusive_scan_u32 (cospanmdao/include/naga/cospan/device_scan.hpp:46-110), a recursive
// reduce-then-scan of 3 kernels per level with temporary allocations, by ONE launch over tiles:
//   1. a tile takes a dynamic tile index (so every tile it waits on has started) and sums its items: 16-byte aligned
//      plain arrays with 16-byte loads kept in L2 (k_scan_l2, 32 KB per 128-thread tile), a column from aligned 32-bit
//      counts with one untiled bulk copy of 24 KB into shared memory (k_column_bulk), other arrays with coalesced
//      loads of 256 threads × ITEMS through shared memory (k_scan);
//   2. it publishes its aggregate (flag 1), then warp 0 looks back over its predecessors 32 at a time (flag and value
//      in one 64-bit word, so one round is one L2 round trip), adding aggregates until it meets a published inclusive
//      prefix (flag 2), and publishes its own inclusive prefix;
//   3. it scans its items from that prefix (k_scan_l2 reads them again, from L2) and writes them coalesced; the last
//      tile writes out[n], the total.
// Integer addition mod 2^32 / 2^64 is associative, so the result is bit-identical to std::exclusive_scan whatever the
// order of the lookback. Every wait is bounded (common.cuh).
//
// cspb_build_column fuses the three other launches of cs::detail::build_column (shape_hook.hpp:265-338) into the same
// kernel: the narrowing of the source values (negative -> flag 1, past 32 bits -> flag 2) happens as the tile loads,
// the running sum is carried in 64 bits so that a total past 2^32 - 1 is known exactly (the reference detects the same
// thing as a decrease of the wrapped u32 offsets), and the last tile writes [total, flag].
#include <cstring>
#include <type_traits>

#include "common.cuh"
#include "mbar.cuh"

namespace cspb {

constexpr int kScanThreads = 256;

template <typename T> struct ScanItems;
template <> struct ScanItems<uint32_t> { static constexpr int N = 16; };
template <> struct ScanItems<uint64_t> { static constexpr int N = 8; };

// Where the items come from. Plain: in[i]. Column: narrowed count values of src[i * k] of an integer dtype.
struct ScanSrc {
    const void* in;
    int32_t dtype;  // CSPB_U32 / CSPB_U64 for a plain scan; CSPB_I32/U32/I64/U64 for a column
    int64_t k;      // column stride (build_column), 1 for a plain scan
    bool column;    // narrow + flags
    uint32_t* extents;  // column: the narrowed values are written here
};

// Item i of the source (always < n), read through the read-only global path: a column source's raw value widened to
// 64 bits, a plain source's value.
template <typename T>
__device__ __forceinline__ T load_plain(const ScanSrc& s, int64_t i) {
    return __ldg(static_cast<const T*>(s.in) + i);
}
__device__ __forceinline__ uint64_t load_column(const ScanSrc& s, int64_t i) {
    switch (s.dtype) {
        case CSPB_I32: return uint64_t(int64_t(__ldg(static_cast<const int32_t*>(s.in) + i * s.k)));
        case CSPB_U32: return uint64_t(__ldg(static_cast<const uint32_t*>(s.in) + i * s.k));
        case CSPB_I64: return uint64_t(__ldg(reinterpret_cast<const long long*>(s.in) + i * s.k));
        default: return uint64_t(__ldg(reinterpret_cast<const unsigned long long*>(s.in) + i * s.k));
    }
}
// A column value narrowed to u32 (cs::detail::build_column's rule): negative -> 0 and flag 1, past 32 bits -> 0 and
// flag 2 (the signed dtypes were sign-extended by load_column).
__device__ __forceinline__ uint32_t narrow(int32_t dtype, uint64_t raw, uint32_t& flag) {
    const bool sgn = dtype == CSPB_I32 || dtype == CSPB_I64;
    if (sgn && int64_t(raw) < 0) {
        flag |= 1u;
        return 0u;
    }
    if (raw > 0xffffffffull) {
        flag |= 2u;
        return 0u;
    }
    return uint32_t(raw);
}

template <typename T>
struct ScanK {
    ScanSrc src;
    T* out;             // n + 1 (column: u32 offsets, T = u64 carries the exact running sum)
    uint32_t* out32;    // column mode: the u32 offsets are written here instead of out
    int64_t n;
    int64_t tiles;
    uint32_t* ctrl;
    uint64_t* tstat;    // per tile: its status words (TileStat<T>)
    uint32_t* total_flag;  // column mode: [total, flag]
    uint64_t* total64;     // a column with u64 offsets: its total (its flag word is total_flag)
};

// A tile's published state: flag (0 nothing, 1 aggregate, 2 inclusive prefix) and value in single 64-bit words, so a
// reader gets both with one load and needs no fence between them. u32: one word, flag in the high half. u64: two
// words (the value's low and high halves), each with the flag in its high half; a reader takes the pair only when both
// flags agree (a pair caught between two stores is read again).
template <typename T> struct TileStat;
template <> struct TileStat<uint32_t> {
    static constexpr int kWords = 1;
    static __device__ __forceinline__ void put(uint64_t* w, uint32_t flag, uint32_t v) {
        st_relaxed64(w, (uint64_t(flag) << 32) | v);
    }
    static __device__ __forceinline__ uint32_t get(const uint64_t* w, uint32_t& v) {
        const uint64_t a = ld_relaxed64(w);
        v = uint32_t(a);
        return uint32_t(a >> 32);
    }
};
template <> struct TileStat<uint64_t> {
    static constexpr int kWords = 2;
    static __device__ __forceinline__ void put(uint64_t* w, uint32_t flag, uint64_t v) {
        st_relaxed64(w, (uint64_t(flag) << 32) | (v & 0xffffffffull));
        st_relaxed64(w + 1, (uint64_t(flag) << 32) | (v >> 32));
    }
    static __device__ __forceinline__ uint32_t get(const uint64_t* w, uint64_t& v) {
        const uint64_t a = ld_relaxed64(w), b = ld_relaxed64(w + 1);
        v = (b << 32) | (a & 0xffffffffull);
        const uint32_t fa = uint32_t(a >> 32), fb = uint32_t(b >> 32);
        return fa == fb ? fa : 0u;
    }
};

// Predecessors each lane of the looking-back warp reads per round: one round covers 32·kLook tiles. One tile a lane
// (32 a round) is the fastest on B200 at 2^28 u32 items: 0.76 ms against 0.81 (2 a lane), 0.95 (4) and 1.33 (8), at 6
// blocks per SM. A round's status words are the lines every looking-back warp polls, and a round of 256 tiles (16
// lines) made each poll several times slower than the walk back it saved.
template <typename T> inline constexpr int kLook = 1;

template <typename T>
__device__ __forceinline__ T warp_incl_scan(T v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const T o = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += o;
    }
    return v;
}

// Warp 0 of a tile: publishes the tile's aggregate (flag 1), looks back over its predecessors until a published
// inclusive prefix, publishes its own inclusive prefix (flag 2) and leaves the tile's exclusive prefix in *s_prefix.
// Every wait is bounded: a wait that gives up sets CSPB_DEV_TIMEOUT (and, for a column, the flag word's timeout bit).
template <typename T>
__device__ __forceinline__ void tile_lookback(const ScanK<T>& g, uint32_t tile, T agg, T* s_prefix) {
    const int lane = threadIdx.x & 31;
    using TS = TileStat<T>;
    constexpr int W = TS::kWords;
    constexpr int kLook = cspb::kLook<T>;
    if (tile == 0) {
        if (lane == 0) {
            TS::put(g.tstat, 2u, agg);
            *s_prefix = 0;
        }
    } else {
        if (lane == 0) TS::put(g.tstat + int64_t(tile) * W, 1u, agg);
        T prefix = 0;
        int64_t base = int64_t(tile) - 1;  // the nearest predecessor of this round
        const unsigned long long t0 = globaltimer_ns();
        bool done = false, gave_up = false;
        while (!done) {
            // lane l reads predecessors base - (l·kLook + j), j = 0 .. kLook-1 (lane 0 the nearest); a
            // predecessor before tile 0 reads as an inclusive prefix of 0
            uint32_t f[kLook];
            T v[kLook];
            int first, stop;
            for (;;) {
#pragma unroll
                for (int j = 0; j < kLook; ++j) {
                    const int64_t p = base - (lane * kLook + j);
                    if (p >= 0) f[j] = TS::get(g.tstat + p * W, v[j]);
                    else { f[j] = 2u; v[j] = T(0); }
                }
                first = kLook;  // this lane's nearest inclusive prefix
                bool zero = false;
#pragma unroll
                for (int j = kLook - 1; j >= 0; --j)
                    if (f[j] == 2u) first = j;
#pragma unroll
                for (int j = 0; j < kLook; ++j)
                    if (j < first && f[j] == 0u) zero = true;
                const unsigned incl = __ballot_sync(0xffffffffu, first < kLook);
                stop = incl ? __ffs(incl) - 1 : 32;  // the lane holding the nearest inclusive prefix
                // every predecessor up to that prefix must have published at least its aggregate
                const bool wait = lane <= stop && zero;
                if (!__any_sync(0xffffffffu, wait)) break;
                int give_up = 0;
                if (lane == 0) {
                    if (status_timed_out(g.ctrl)) give_up = 1;
                    else if (globaltimer_ns() - t0 > kWaitBudgetNs) {
                        set_status(g.ctrl, CSPB_DEV_TIMEOUT);
                        // a column build also reports it beside its other flags: a caller without the
                        // workspace (cspb_build_column_static) has no other way to see it
                        if (g.total_flag) atomicOr(g.total_flag + 1, CSPB_COLUMN_TIMEOUT);
                        give_up = 1;
                    }
                }
                if (__shfl_sync(0xffffffffu, give_up, 0)) {
                    gave_up = true;
                    break;
                }
                __nanosleep(32);
            }
            if (gave_up) break;
            T c = 0;
            if (lane < stop) {
#pragma unroll
                for (int j = 0; j < kLook; ++j) c += v[j];
            } else if (lane == stop) {
#pragma unroll
                for (int j = 0; j < kLook; ++j)
                    if (j <= first) c += v[j];
            }
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
            prefix += c;
            if (stop < 32) done = true;
            else base -= 32 * kLook;
        }
        if (lane == 0) {
            if (!gave_up) TS::put(g.tstat + int64_t(tile) * W, 2u, prefix + agg);
            *s_prefix = prefix;
        }
    }
}

// Where a tile's items come from: a plain array, or a column's count values of a 32-bit or a 64-bit dtype.
enum ScanMode : int { kPlain = 0, kColumn32 = 1, kColumn64 = 2 };

// A column value of a 32-bit dtype, kept in 32 bits until it is narrowed (a signed value is sign-extended then).
__device__ __forceinline__ uint32_t load_column32(const ScanSrc& s, int64_t i) {
    return __ldg(static_cast<const uint32_t*>(s.in) + i * s.k);
}
__device__ __forceinline__ uint64_t widen_column32(int32_t dtype, uint32_t raw) {
    return dtype == CSPB_I32 ? uint64_t(int64_t(int32_t(raw))) : uint64_t(raw);
}

// 8 blocks per SM (32 registers) for the plain and the 32-bit column tiles: the whole SM's warp slots hold tiles, and a
// tile spends most of its life in the look-back, so the tiles resident decide the bytes in flight (2^28 u32: 0.67 ms
// against 0.76 ms at 6 blocks). A 64-bit column tile holds 16 raw 64-bit values in flight: 6 blocks.
template <typename T, int MODE>
__global__ void __launch_bounds__(kScanThreads, MODE == kColumn64 ? 6 : 8) k_scan(ScanK<T> g) {
    constexpr int IT = ScanItems<T>::N;
    constexpr int TILE = kScanThreads * IT;
    constexpr int PAD = TILE + TILE / 32;
    __shared__ T sm[PAD];
    __shared__ T s_warp[kScanThreads / 32];
    __shared__ T s_prefix;
    __shared__ uint32_t s_flag;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;

    const uint32_t tile = grab_work(g.ctrl, kWork0);
    if (tile >= g.tiles) return;
    if (t == 0) s_flag = 0;
    const int64_t base = int64_t(tile) * TILE;

    // 1. striped coalesced load -> shared (padded) -> blocked items. Every load of the tile is issued before the first
    // store: the loads go through the read-only global path into registers, then the stores follow (a load through a
    // generic pointer, stored to shared memory in the same loop, could not be moved past the previous store).
    uint32_t flag = 0;
    if constexpr (MODE == kPlain) {
        T x[IT];
#pragma unroll
        for (int k = 0; k < IT; ++k) {
            const int64_t i = base + k * kScanThreads + t;
            x[k] = i < g.n ? load_plain<T>(g.src, i) : T(0);
        }
#pragma unroll
        for (int k = 0; k < IT; ++k) {
            const int idx = k * kScanThreads + t;
            sm[idx + idx / 32] = x[k];
        }
    } else {
        using Raw = std::conditional_t<MODE == kColumn32, uint32_t, uint64_t>;
        Raw raw[IT];
#pragma unroll
        for (int k = 0; k < IT; ++k) {
            const int64_t i = base + k * kScanThreads + t;
            if constexpr (MODE == kColumn32) raw[k] = i < g.n ? load_column32(g.src, i) : 0u;
            else raw[k] = i < g.n ? load_column(g.src, i) : 0ull;
        }
#pragma unroll
        for (int k = 0; k < IT; ++k) {
            const int idx = k * kScanThreads + t;
            const int64_t i = base + idx;
            uint32_t x = 0;
            if (i < g.n) {
                if constexpr (MODE == kColumn32) x = narrow(g.src.dtype, widen_column32(g.src.dtype, raw[k]), flag);
                else x = narrow(g.src.dtype, raw[k], flag);
                __stcg(g.src.extents + i, x);
            }
            sm[idx + idx / 32] = T(x);
        }
    }
    __syncthreads();
    if (flag) atomicOr(&s_flag, flag);
    T v[IT];
    T run = 0;
#pragma unroll
    for (int k = 0; k < IT; ++k) {
        const int idx = t * IT + k;
        v[k] = run;  // exclusive within the thread
        run += sm[idx + idx / 32];
    }
    // block scan of the thread totals
    const T incl = warp_incl_scan(run);
    if (lane == 31) s_warp[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        T wv = lane < kScanThreads / 32 ? s_warp[lane] : T(0);
        const T wi = warp_incl_scan(wv);
        if (lane < kScanThreads / 32) s_warp[lane] = wi - wv;  // exclusive warp offsets
    }
    __syncthreads();
    const T thread_excl = s_warp[warp] + incl - run;
    __shared__ T s_agg;
    if (t == kScanThreads - 1) s_agg = thread_excl + run;
    // the tile's exclusive values wait in shared memory (blocked order) during the look-back, not in registers (every
    // thread's last read of sm was before the barriers above)
#pragma unroll
    for (int k = 0; k < IT; ++k) {
        const int idx = t * IT + k;
        sm[idx + idx / 32] = thread_excl + v[k];
    }
    __syncthreads();
    const T agg = s_agg;

    // 2. publish the aggregate, look back, publish the inclusive prefix
    if (warp == 0) tile_lookback<T>(g, tile, agg, &s_prefix);
    __syncthreads();
    const T prefix = s_prefix;

    // 3. the tile's prefix plus its exclusive values, from shared memory in striped order: coalesced stores
#pragma unroll
    for (int k = 0; k < IT; ++k) {
        const int idx = k * kScanThreads + t;
        const int64_t i = base + idx;
        if (i < g.n) {
            const T o = prefix + sm[idx + idx / 32];
            if (g.out32) __stcg(g.out32 + i, uint32_t(o));
            else __stcg(g.out + i, o);
        }
    }
    if (s_flag && t == 0) {
        if (g.total_flag) atomicOr(g.total_flag + 1, s_flag);
        set_status(g.ctrl, ((s_flag & 1u) ? CSPB_DEV_NEGATIVE : 0u) | ((s_flag & 2u) ? CSPB_DEV_EXCEEDS32 : 0u));
    }
    if (tile == g.tiles - 1 && t == 0) {
        const T total = prefix + agg;
        if (g.out32) {
            g.out32[g.n] = uint32_t(total);
            if (g.total_flag) {
                const bool over = uint64_t(total) > 0xffffffffull;
                g.total_flag[0] = uint32_t(total);
                if (over) {
                    atomicOr(g.total_flag + 1, 2u);
                    set_status(g.ctrl, CSPB_DEV_EXCEEDS32);
                }
            }
        } else {
            g.out[g.n] = total;
            if (g.total64) g.total64[0] = uint64_t(total);
        }
    }
}

// ---- bulk tiles: build_column from 16-byte aligned 32-bit counts ----------------------------------------------------
// A tile of 128 threads arrives with ONE untiled bulk copy (TMA) of 24 KB into shared memory: no registers hold loads
// in flight, so 9 tiles fit an SM (216 KB), and a tile in its look-back holds only shared memory. Pass 1 narrows and
// sums each warp's 12 rows (a row = 32 lanes × 16 bytes, read conflict-free), warp 0 looks back with the tile's
// aggregate, and pass 2 scans the rows again from the tile's prefix and stores them with 16-byte stores. 2^28 i32
// counts: 0.587 ms (84 % of the measured copy bandwidth; it writes twice the bytes it reads). The plain scans took
// these tiles too (2^28 u32: 0.512 ms) before the L2 re-read tiles below.
constexpr int kBulkThreads = 128;
constexpr int kBulkRows = 12;  // rows per warp
template <typename T> struct BulkTile {
    static constexpr int kVec = 16 / int(sizeof(T));              // items in a 16-byte vector
    static constexpr int kItems = 4 * kBulkRows * 32 * kVec;      // 6144 u32 / 3072 u64
    static constexpr uint32_t kBytes = uint32_t(kItems * sizeof(T));  // 24 KB
};

template <typename T> struct Vec16;
template <> struct Vec16<uint32_t> {
    static __device__ __forceinline__ void unpack(const uint4& v, uint32_t (&x)[4]) {
        x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
    }
    static __device__ __forceinline__ void store(uint32_t* p, const uint32_t (&o)[4]) {
        asm volatile("st.global.cg.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(o[0]), "r"(o[1]), "r"(o[2]), "r"(o[3])
                     : "memory");
    }
};
template <> struct Vec16<uint64_t> {
    static __device__ __forceinline__ void unpack(const uint4& v, uint64_t (&x)[2]) {
        x[0] = (uint64_t(v.y) << 32) | v.x;
        x[1] = (uint64_t(v.w) << 32) | v.z;
    }
    static __device__ __forceinline__ void store(uint64_t* p, const uint64_t (&o)[2]) {
        asm volatile("st.global.cg.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(o[0]), "l"(o[1]) : "memory");
    }
};

// ---- L2 re-read tiles: the plain scans of 16-byte aligned arrays -----------------------------------------------------
// A tile of 128 threads reads its 32 KB from DRAM once in pass 1 (16-byte loads kept in L2 with an evict-last policy)
// and sums it, warp 0 looks back with the tile's aggregate, and pass 2 reads the tile again (from L2, evict-first) and
// scans and stores it. The tile holds no shared memory while it waits in the look-back, so 12 tiles fit an SM (3 ×
// the bytes a bulk-copy tile could hold there) and their DRAM reads stay in flight; ~57 MB of tiles sit in L2 at a
// time. 2^28 u32 items: 0.441 ms against 0.512 ms for the bulk-copy tiles and 0.52 ms for the same tiles without the
// L2 policies.
constexpr int kL2Threads = 128;
constexpr int kL2Rows = 16;   // rows of 32 lanes × 16 bytes per warp
constexpr int kL2Flight = 4;  // rows each lane keeps in flight
template <typename T> struct L2Tile {
    static constexpr int kVec = 16 / int(sizeof(T));
    static constexpr int kItems = 4 * kL2Rows * 32 * kVec;  // 8192 u32 / 4096 u64
};

__device__ __forceinline__ uint4 ld_policy_u4(const void* p, uint64_t pol) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p), "l"(pol));
    return v;
}
__device__ __forceinline__ uint64_t evict_last_l2_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
template <typename T> struct VecCs;
template <> struct VecCs<uint32_t> {
    static __device__ __forceinline__ void store(uint32_t* p, const uint32_t (&o)[4]) {
        asm volatile("st.global.cs.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(o[0]), "r"(o[1]), "r"(o[2]), "r"(o[3])
                     : "memory");
    }
};
template <> struct VecCs<uint64_t> {
    static __device__ __forceinline__ void store(uint64_t* p, const uint64_t (&o)[2]) {
        asm volatile("st.global.cs.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(o[0]), "l"(o[1]) : "memory");
    }
};

// A row of the tile as one 16-byte vector per lane: the whole vector when the tile is full, else element by element
// (zero past n).
template <typename T>
__device__ __forceinline__ uint4 l2_row(const T* in, int64_t i0, int64_t n, bool full, uint64_t pol) {
    if (full) return ld_policy_u4(in + i0, pol);
    constexpr int E = 16 / int(sizeof(T));
    T x[E];
#pragma unroll
    for (int k = 0; k < E; ++k) x[k] = i0 + k < n ? __ldg(in + i0 + k) : T(0);
    uint4 v;
    memcpy(&v, x, 16);
    return v;
}

template <typename T>
__global__ void __launch_bounds__(kL2Threads, 12) k_scan_l2(ScanK<T> g) {
    constexpr int E = L2Tile<T>::kVec;
    constexpr int TILE = L2Tile<T>::kItems;
    constexpr int B = kL2Flight;
    __shared__ T s_wsum[4];
    __shared__ T s_prefix;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const uint32_t tile = grab_work(g.ctrl, kWork0);
    if (tile >= g.tiles) return;
    const int64_t base = int64_t(tile) * TILE;
    const bool full = g.n - base >= TILE;
    const T* in = static_cast<const T*>(g.src.in);
    const uint64_t keep = evict_last_l2_policy(), drop = evict_first_policy();
    // pass 1: the warp's sum, its rows kept in L2
    T s = 0;
#pragma unroll
    for (int j0 = 0; j0 < kL2Rows; j0 += B) {
        uint4 v[B];
#pragma unroll
        for (int k = 0; k < B; ++k)
            v[k] = l2_row<T>(in, base + int64_t(warp * kL2Rows + j0 + k) * 32 * E + lane * E, g.n, full, keep);
#pragma unroll
        for (int k = 0; k < B; ++k) {
            T x[E];
            Vec16<T>::unpack(v[k], x);
#pragma unroll
            for (int q = 0; q < E; ++q) s += x[q];
        }
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) s_wsum[warp] = s;
    __syncthreads();
    const T agg = (s_wsum[0] + s_wsum[1]) + (s_wsum[2] + s_wsum[3]);
    if (warp == 0) tile_lookback<T>(g, tile, agg, &s_prefix);
    __syncthreads();
    // pass 2: the rows again (from L2), scanned from the tile's prefix plus the sums of the warps before
    T carry = s_prefix;
#pragma unroll
    for (int w = 0; w < 3; ++w)
        if (w < warp) carry += s_wsum[w];
    T* out = g.out;
#pragma unroll
    for (int j0 = 0; j0 < kL2Rows; j0 += B) {
        uint4 v[B];
#pragma unroll
        for (int k = 0; k < B; ++k)
            v[k] = l2_row<T>(in, base + int64_t(warp * kL2Rows + j0 + k) * 32 * E + lane * E, g.n, full, drop);
#pragma unroll
        for (int k = 0; k < B; ++k) {
            T x[E];
            Vec16<T>::unpack(v[k], x);
            T c[E];
            c[0] = x[0];
#pragma unroll
            for (int q = 1; q < E; ++q) c[q] = c[q - 1] + x[q];
            const T inc = warp_incl_scan(c[E - 1]);
            const T e = carry + inc - c[E - 1];
            carry += __shfl_sync(0xffffffffu, inc, 31);
            T o[E];
            o[0] = e;
#pragma unroll
            for (int q = 1; q < E; ++q) o[q] = e + c[q - 1];
            const int64_t i0 = base + int64_t(warp * kL2Rows + j0 + k) * 32 * E + lane * E;
            if (full) {
                VecCs<T>::store(out + i0, o);
            } else {
#pragma unroll
                for (int q = 0; q < E; ++q)
                    if (i0 + q < g.n) __stcg(out + i0 + q, o[q]);
            }
        }
    }
    if (tile == g.tiles - 1 && t == kL2Threads - 1) out[g.n] = carry;  // the total
}

// Counts mode of build_column on bulk tiles: a 32-bit count source with stride 1. Pass 1 narrows the counts (a
// negative i32 is 0 and flag 1), writes the extents and the narrowed values back to the tile, and sums them in 64 bits;
// pass 2 scans them from the tile's prefix into u32 offsets (out32) or u64 offsets (out). The extents, the offsets and
// the flags are those of k_scan's column mode.
template <bool SIGNED>
__global__ void __launch_bounds__(kBulkThreads, 9) k_column_bulk(ScanK<uint64_t> g) {
    constexpr int TILE = BulkTile<uint32_t>::kItems;
    extern __shared__ __align__(128) unsigned char dsm[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint64_t s_wsum[4];
    __shared__ uint64_t s_prefix;
    __shared__ uint32_t s_flag;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) {
        mbar_init(&bar, 1);
        fence_mbar_init();
        s_flag = 0;
    }
    const uint32_t tile = grab_work(g.ctrl, kWork0);
    if (tile >= g.tiles) return;
    const int64_t base = int64_t(tile) * TILE;
    const int64_t cnt = g.n - base < TILE ? g.n - base : TILE;
    const uint32_t* in = static_cast<const uint32_t*>(g.src.in);
    if (cnt == TILE) {
        if (t == 0) {
            mbar_arrive_tx(&bar, BulkTile<uint32_t>::kBytes);
            bulk_load_1d(dsm, in + base, BulkTile<uint32_t>::kBytes, &bar);
        }
        if (!mbar_wait_own_copy(&bar, 0)) {
            set_status(g.ctrl, CSPB_DEV_TIMEOUT);
            if (g.total_flag) atomicOr(g.total_flag + 1, CSPB_COLUMN_TIMEOUT);
            return;
        }
    } else {
        uint32_t* b32 = reinterpret_cast<uint32_t*>(dsm);
        for (int i = t; i < TILE; i += kBulkThreads) b32[i] = i < cnt ? __ldg(in + base + i) : 0u;
        __syncthreads();
    }
    uint4* buf = reinterpret_cast<uint4*>(dsm);
    uint32_t* ext = g.src.extents;
    // pass 1: narrow, extents, the warp's sum
    uint64_t s = 0;
    uint32_t flag = 0;
#pragma unroll 4
    for (int j = 0; j < kBulkRows; ++j) {
        const int row = warp * kBulkRows + j;
        uint4 v = buf[row * 32 + lane];
        if constexpr (SIGNED) {
            const auto nz = [&flag](uint32_t x) {
                if (int32_t(x) < 0) {
                    flag |= 1u;
                    return 0u;
                }
                return x;
            };
            v.x = nz(v.x);
            v.y = nz(v.y);
            v.z = nz(v.z);
            v.w = nz(v.w);
            buf[row * 32 + lane] = v;
        }
        const int64_t i0 = base + int64_t(row) * 128 + lane * 4;
        if (cnt == TILE) {
            asm volatile("st.global.cg.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(ext + i0), "r"(v.x), "r"(v.y), "r"(v.z),
                         "r"(v.w)
                         : "memory");
        } else {
            const uint32_t o4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (i0 + k < g.n) __stcg(ext + i0 + k, o4[k]);
        }
        s += (uint64_t(v.x) + v.y) + (uint64_t(v.z) + v.w);
    }
    if (flag) atomicOr(&s_flag, flag);
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) s_wsum[warp] = s;
    __syncthreads();
    const uint64_t agg = (s_wsum[0] + s_wsum[1]) + (s_wsum[2] + s_wsum[3]);
    if (warp == 0) tile_lookback<uint64_t>(g, tile, agg, &s_prefix);
    __syncthreads();
    // pass 2: the offsets
    uint64_t carry = s_prefix;
#pragma unroll
    for (int w = 0; w < 3; ++w)
        if (w < warp) carry += s_wsum[w];
#pragma unroll
    for (int j = 0; j < kBulkRows; ++j) {
        const int row = warp * kBulkRows + j;
        const uint4 v = buf[row * 32 + lane];
        const uint64_t c0 = v.x, c1 = c0 + v.y, c2 = c1 + v.z, c3 = c2 + v.w;
        const uint64_t inc = warp_incl_scan(c3);
        const uint64_t e = carry + inc - c3;
        carry += __shfl_sync(0xffffffffu, inc, 31);
        const uint64_t o[4] = {e, e + c0, e + c1, e + c2};
        const int64_t i0 = base + int64_t(row) * 128 + lane * 4;
        if (cnt == TILE) {
            if (g.out32) {
                asm volatile("st.global.cg.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(g.out32 + i0), "r"(uint32_t(o[0])),
                             "r"(uint32_t(o[1])), "r"(uint32_t(o[2])), "r"(uint32_t(o[3]))
                             : "memory");
            } else {
                asm volatile("st.global.cg.v2.u64 [%0], {%1, %2};" ::"l"(g.out + i0), "l"(o[0]), "l"(o[1]) : "memory");
                asm volatile("st.global.cg.v2.u64 [%0], {%1, %2};" ::"l"(g.out + i0 + 2), "l"(o[2]), "l"(o[3])
                             : "memory");
            }
        } else {
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (i0 + k < g.n) {
                    if (g.out32) __stcg(g.out32 + i0 + k, uint32_t(o[k]));
                    else __stcg(g.out + i0 + k, o[k]);
                }
        }
    }
    __syncthreads();  // every thread's flag is in s_flag
    if (s_flag && t == 0) {
        if (g.total_flag) atomicOr(g.total_flag + 1, s_flag);
        set_status(g.ctrl, CSPB_DEV_NEGATIVE);
    }
    if (tile == g.tiles - 1 && t == kBulkThreads - 1) {
        const uint64_t total = carry;
        if (g.out32) {
            g.out32[g.n] = uint32_t(total);
            if (g.total_flag) {
                g.total_flag[0] = uint32_t(total);
                if (total > 0xffffffffull) {
                    atomicOr(g.total_flag + 1, 2u);
                    set_status(g.ctrl, CSPB_DEV_EXCEEDS32);
                }
            }
        } else {
            g.out[g.n] = total;
            if (g.total64) g.total64[0] = total;
        }
    }
}

// Offsets mode of build_column: offs[i] = narrowed value (bad: negative, offs[0] != 0), extents from differences.
__global__ void k_column_offsets(ScanSrc s, int64_t m, uint32_t* offs, uint32_t* ctrl, uint32_t* total_flag) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
        uint32_t flag = 0, x = 0;
        switch (s.dtype) {
            case CSPB_I32: { const int32_t v = static_cast<const int32_t*>(s.in)[i]; if (v < 0) flag |= 1u; else x = uint32_t(v); break; }
            case CSPB_U32: x = static_cast<const uint32_t*>(s.in)[i]; break;
            case CSPB_I64: {
                const int64_t v = static_cast<const int64_t*>(s.in)[i];
                if (v < 0) flag |= 1u; else if (v > int64_t(0xffffffffll)) flag |= 2u; else x = uint32_t(v);
                break;
            }
            default: { const uint64_t v = static_cast<const uint64_t*>(s.in)[i]; if (v > 0xffffffffull) flag |= 2u; else x = uint32_t(v); break; }
        }
        if (i == 0 && x != 0) flag |= 1u;
        offs[i] = x;
        if (flag) {
            atomicOr(total_flag + 1, flag);
            set_status(ctrl, ((flag & 1u) ? CSPB_DEV_NEGATIVE : 0u) | ((flag & 2u) ? CSPB_DEV_EXCEEDS32 : 0u));
        }
    }
}
__global__ void k_column_extents(const uint32_t* offs, int64_t n, uint32_t* extents, uint32_t* ctrl, uint32_t* total_flag) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t a = offs[i], b = offs[i + 1];
        if (b < a) {
            extents[i] = 0;
            atomicOr(total_flag + 1, 1u);
            set_status(ctrl, CSPB_DEV_NEGATIVE);
        } else {
            extents[i] = b - a;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) total_flag[0] = offs[n];
}

// Offsets mode with u64 offsets: the values need not fit 32 bits; each extent (a difference) still must.
__global__ void k_column_offsets64(ScanSrc s, int64_t m, uint64_t* offs, uint32_t* ctrl, uint32_t* flagw) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < m; i += stride) {
        const uint64_t raw = load_column(s, i);
        const bool sgn = s.dtype == CSPB_I32 || s.dtype == CSPB_I64;
        uint64_t x = raw;
        uint32_t flag = 0;
        if (sgn && int64_t(raw) < 0) {
            flag = 1u;
            x = 0;
        }
        if (i == 0 && x != 0) flag |= 1u;
        offs[i] = x;
        if (flag) {
            atomicOr(flagw, flag);
            set_status(ctrl, CSPB_DEV_NEGATIVE);
        }
    }
}
__global__ void k_column_extents64(const uint64_t* offs, int64_t n, uint32_t* extents, uint32_t* ctrl,
                                   uint32_t* flagw, uint64_t* total64) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint64_t a = offs[i], b = offs[i + 1];
        uint32_t flag = 0;
        if (b < a) flag = 1u;
        else if (b - a > 0xffffffffull) flag = 2u;
        extents[i] = flag ? 0u : uint32_t(b - a);
        if (flag) {
            atomicOr(flagw, flag);
            set_status(ctrl, flag == 1u ? CSPB_DEV_NEGATIVE : CSPB_DEV_EXCEEDS32);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) total64[0] = offs[n];
}

__global__ void k_scan_empty32(uint32_t* out) { out[0] = 0; }
__global__ void k_scan_empty64(uint64_t* out) { out[0] = 0; }

}  // namespace cspb

using namespace cspb;
using cspb_host::align_up;
using cspb_host::aligned;

namespace {

template <typename T>
struct ScanLayout {
    int64_t tiles = 0;
    size_t off_stat = 0, total = 0;
};

template <typename T>
ScanLayout<T> scan_layout(int64_t n) {
    ScanLayout<T> L;
    const int64_t TILE = int64_t(kScanThreads) * ScanItems<T>::N;
    L.tiles = n <= 0 ? 0 : (n + TILE - 1) / TILE;
    L.off_stat = kCtrlBytes;
    L.total = align_up(kCtrlBytes + size_t(L.tiles) * 8 * TileStat<T>::kWords, 256);
    return L;
}

template <typename T>
int run_scan(const ScanSrc& src, T* out, uint32_t* out32, int64_t n, void* ws, size_t ws_bytes, uint32_t* total_flag,
             cudaStream_t st, uint64_t* total64 = nullptr) {
    const ScanLayout<T> L = scan_layout<T>(n);
    if (!ws || !aligned(ws, 256) || ws_bytes < L.total) return CSPB_ERR_WORKSPACE;
    char* w = static_cast<char*>(ws);
    cudaError_t e = cudaMemsetAsync(w, 0, L.total, st);  // ctrl + tile status words
    if (e != cudaSuccess) return CSPB_ERR_CUDA;
    ScanK<T> g{};
    g.src = src;
    g.out = out;
    g.out32 = out32;
    g.n = n;
    g.tiles = L.tiles;
    g.ctrl = reinterpret_cast<uint32_t*>(w);
    g.tstat = reinterpret_cast<uint64_t*>(w + L.off_stat);
    g.total_flag = total_flag;
    g.total64 = total64;
    if (!src.column && aligned(src.in, 16) && aligned(out, 16)) {
        // L2 re-read tiles (fewer, larger tiles than the layout's: the layout's status words cover them)
        g.tiles = (n + L2Tile<T>::kItems - 1) / L2Tile<T>::kItems;
        k_scan_l2<T><<<unsigned(g.tiles), kL2Threads, 0, st>>>(g);
    } else if (!src.column) k_scan<T, kPlain><<<unsigned(L.tiles), kScanThreads, 0, st>>>(g);
    else if constexpr (std::is_same_v<T, uint64_t>) {
        if ((src.dtype == CSPB_I32 || src.dtype == CSPB_U32) && src.k == 1 && aligned(src.in, 16) &&
            aligned(src.extents, 16) && aligned(out32 ? static_cast<const void*>(out32) : out, 16)) {
            g.tiles = (n + BulkTile<uint32_t>::kItems - 1) / BulkTile<uint32_t>::kItems;
            if (src.dtype == CSPB_I32)
                k_column_bulk<true><<<unsigned(g.tiles), kBulkThreads, BulkTile<uint32_t>::kBytes, st>>>(g);
            else k_column_bulk<false><<<unsigned(g.tiles), kBulkThreads, BulkTile<uint32_t>::kBytes, st>>>(g);
        } else if (src.dtype == CSPB_I32 || src.dtype == CSPB_U32)
            k_scan<T, kColumn32><<<unsigned(L.tiles), kScanThreads, 0, st>>>(g);
        else k_scan<T, kColumn64><<<unsigned(L.tiles), kScanThreads, 0, st>>>(g);
    } else if (src.dtype == CSPB_I32 || src.dtype == CSPB_U32)
        k_scan<T, kColumn32><<<unsigned(L.tiles), kScanThreads, 0, st>>>(g);
    else k_scan<T, kColumn64><<<unsigned(L.tiles), kScanThreads, 0, st>>>(g);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

}  // namespace

extern "C" {

size_t cspb_scan_workspace_bytes(int64_t n) {
    if (n < 0) return 0;
    const size_t a = scan_layout<uint32_t>(n).total, b = scan_layout<uint64_t>(n).total;
    return a > b ? a : b;
}

int cspb_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, void* workspace, size_t workspace_bytes,
                            void* stream) {
    if (n < 0 || !out || (n > 0 && !in)) return CSPB_ERR_ARGUMENT;
    if (n > (int64_t(1) << 40)) return CSPB_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        k_scan_empty32<<<1, 1, 0, st>>>(out);
        return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
    }
    ScanSrc s{in, CSPB_U32, 1, false, nullptr};
    return run_scan<uint32_t>(s, out, nullptr, n, workspace, workspace_bytes, nullptr, st);
}

int cspb_exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n, void* workspace, size_t workspace_bytes,
                            void* stream) {
    if (n < 0 || !out || (n > 0 && !in)) return CSPB_ERR_ARGUMENT;
    if (n > (int64_t(1) << 40)) return CSPB_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        k_scan_empty64<<<1, 1, 0, st>>>(out);
        return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
    }
    ScanSrc s{in, CSPB_U64, 1, false, nullptr};
    return run_scan<uint64_t>(s, out, nullptr, n, workspace, workspace_bytes, nullptr, st);
}

int cspb_build_column(const void* src, int32_t src_dtype, int64_t count, int64_t k, int32_t offsets_mode,
                      uint32_t* extents, uint32_t* offs, uint32_t* total_flag, void* workspace, size_t workspace_bytes,
                      void* stream) {
    if (src_dtype < CSPB_I32 || src_dtype > CSPB_U64) return CSPB_ERR_UNSUPPORTED;
    if (count < 0 || !offs || !total_flag || (count > 0 && !src)) return CSPB_ERR_ARGUMENT;
    if (offsets_mode && count == 0) return CSPB_ERR_ARGUMENT;  // N + 1 >= 1 offsets are needed
    if (!offsets_mode && k < 1) return CSPB_ERR_ARGUMENT;
    if (count > (int64_t(1) << 40)) return CSPB_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = offsets_mode ? count - 1 : count;
    if (n > 0 && !extents) return CSPB_ERR_ARGUMENT;
    if (!workspace || !aligned(workspace, 256) || workspace_bytes < cspb_scan_workspace_bytes(n)) return CSPB_ERR_WORKSPACE;
    cudaError_t e = cudaMemsetAsync(total_flag, 0, 2 * sizeof(uint32_t), st);
    if (e != cudaSuccess) return CSPB_ERR_CUDA;
    ScanSrc s{src, src_dtype, offsets_mode ? 1 : k, true, extents};
    if (!offsets_mode) {
        if (n == 0) {
            e = cudaMemsetAsync(workspace, 0, kCtrlBytes, st);
            if (e != cudaSuccess) return CSPB_ERR_CUDA;
            k_scan_empty32<<<1, 1, 0, st>>>(offs);
            return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
        }
        // the running sum in 64 bits, the offsets stored as u32
        return run_scan<uint64_t>(s, nullptr, offs, n, workspace, workspace_bytes, total_flag, st);
    }
    e = cudaMemsetAsync(workspace, 0, kCtrlBytes, st);
    if (e != cudaSuccess) return CSPB_ERR_CUDA;
    uint32_t* ctrl = static_cast<uint32_t*>(workspace);
    const int64_t blocks = count / 256 + 1 > 1024 ? 1024 : count / 256 + 1;
    k_column_offsets<<<unsigned(blocks), 256, 0, st>>>(s, count, offs, ctrl, total_flag);
    k_column_extents<<<unsigned(blocks), 256, 0, st>>>(offs, n, extents, ctrl, total_flag);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

int cspb_build_column64(const void* src, int32_t src_dtype, int64_t count, int64_t k, int32_t offsets_mode,
                        uint32_t* extents, uint64_t* offs, uint64_t* total_flag, void* workspace,
                        size_t workspace_bytes, void* stream) {
    if (src_dtype < CSPB_I32 || src_dtype > CSPB_U64) return CSPB_ERR_UNSUPPORTED;
    if (count < 0 || !offs || !total_flag || (count > 0 && !src)) return CSPB_ERR_ARGUMENT;
    if (offsets_mode && count == 0) return CSPB_ERR_ARGUMENT;
    if (!offsets_mode && k < 1) return CSPB_ERR_ARGUMENT;
    if (count > (int64_t(1) << 40)) return CSPB_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = offsets_mode ? count - 1 : count;
    if (n > 0 && !extents) return CSPB_ERR_ARGUMENT;
    if (!workspace || !aligned(workspace, 256) || workspace_bytes < cspb_scan_workspace_bytes(n)) return CSPB_ERR_WORKSPACE;
    cudaError_t e = cudaMemsetAsync(total_flag, 0, 2 * sizeof(uint64_t), st);
    if (e != cudaSuccess) return CSPB_ERR_CUDA;
    // the flag word: the low half of total_flag[1] (the same bits as cspb_build_column's total_flag[1])
    uint32_t* flagw = reinterpret_cast<uint32_t*>(total_flag + 1);
    ScanSrc s{src, src_dtype, offsets_mode ? 1 : k, true, extents};
    if (!offsets_mode) {
        if (n == 0) {
            e = cudaMemsetAsync(workspace, 0, kCtrlBytes, st);
            if (e != cudaSuccess) return CSPB_ERR_CUDA;
            k_scan_empty64<<<1, 1, 0, st>>>(offs);
            return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
        }
        // the scan kernel ORs its flags into word 1 of the u32 view it is given: hand it the word before flagw (the
        // high half of the total, which it does not write when it has a 64-bit total)
        return run_scan<uint64_t>(s, offs, nullptr, n, workspace, workspace_bytes, flagw - 1, st, total_flag);
    }
    e = cudaMemsetAsync(workspace, 0, kCtrlBytes, st);
    if (e != cudaSuccess) return CSPB_ERR_CUDA;
    uint32_t* ctrl = static_cast<uint32_t*>(workspace);
    const int64_t blocks = count / 256 + 1 > 1024 ? 1024 : count / 256 + 1;
    k_column_offsets64<<<unsigned(blocks), 256, 0, st>>>(s, count, offs, ctrl, flagw);
    k_column_extents64<<<unsigned(blocks), 256, 0, st>>>(offs, n, extents, ctrl, flagw, total_flag);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

}  // extern "C"

// ---- build_column on a fixed scratch ---------------------------------------------------------------------------------
// The scratch of a u64 scan of CSPB_BUILD_COLUMN_STATIC_MAX items (scan_layout: control block, tile flags, tile
// aggregates, tile prefixes; 2048 items per tile), as a file-scope device array: the call needs no workspace and
// allocates nothing. run_scan / cspb_build_column zero the control block and the tile flags on every call.
namespace {
constexpr int64_t kStaticTiles = (int64_t(CSPB_BUILD_COLUMN_STATIC_MAX) + kScanThreads * ScanItems<uint64_t>::N - 1) /
                                 (kScanThreads * ScanItems<uint64_t>::N);
constexpr size_t kStaticScratchBytes =
    kCtrlBytes + (size_t(kStaticTiles) * 8 * TileStat<uint64_t>::kWords + 255) / 256 * 256;
static_assert(kStaticScratchBytes <= 160 * 1024 + 256, "the fixed scratch stays modest");

static __device__ __align__(256) unsigned char g_column_scratch[kStaticScratchBytes];

// The device address of g_column_scratch in the current device's context. The name is only a host-side stand-in, so
// the address is asked for on every call rather than cached: after a cudaDeviceReset (or under another context) a
// cached address would point at memory that no longer exists. The first call with a device current loads this
// library's device image on that device, which is why it belongs before any stream capture; later lookups are a
// table read.
int column_scratch(void** out) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_column_scratch) != cudaSuccess || !p) return CSPB_ERR_CUDA;
    *out = p;
    return CSPB_OK;
}
}  // namespace

extern "C" int cspb_build_column_static(const void* src, int32_t src_dtype, int64_t count, int64_t k,
                                        int32_t offsets_mode, uint32_t* extents, uint32_t* offs, uint32_t* total_flag,
                                        void* stream) {
    const int64_t n = offsets_mode ? count - 1 : count;
    if (n > int64_t(CSPB_BUILD_COLUMN_STATIC_MAX)) return CSPB_ERR_TOO_LARGE;
    void* scratch = nullptr;
    const int rc = column_scratch(&scratch);
    if (rc != CSPB_OK) return rc;
    return cspb_build_column(src, src_dtype, count, k, offsets_mode, extents, offs, total_flag, scratch,
                             kStaticScratchBytes, stream);
}
