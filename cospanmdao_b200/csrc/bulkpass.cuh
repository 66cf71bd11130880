// bulkpass.cuh — the row pass of rowpass.cuh fed by bulk asynchronous copies into a shared-memory ring.
//
// A CTA is 8 consumer warps (threads 0..255, the warp layout of pass_unit) plus one producer warp (warp 8). The
// producer cuts each unit (S = 128 rows × CW columns) into 4 STAGES of 32 rows: stage s holds rows wy·32 + 8s .. +7 of
// every warp row wy, i.e. exactly the rows a consumer warp handles in pass_unit's batch kb = 8s. Each row segment
// (CW elements = 1 KB) is one cp.async.bulk global→shared copy issued by one producer lane; the stage also carries
// the row vectors of its 32 rows and, in a unit's first stage, the column vectors of the unit's chunk (small copies
// of 16 .. 2048 bytes). All copies of a stage complete on the stage's FULL mbarrier (expect_tx = the stage's bytes);
// the consumers release the stage on its EMPTY mbarrier (one arrival per warp) and the producer refills it. With NST stages in the ring a CTA
// keeps up to NST·32 KB of the matrix in flight while its consumers work, instead of the 8 rows per lane a register
// pipeline can hold.
//
// The consumers compute exactly what pass_unit computes, in the same order (the same unpack, rank-2 update, f64
// column accumulation over the warp's rows in index order, row dots, and the shared unit_epilogue), so a result is
// bit-identical to the register path's. Waits are bounded: one consumer thread waits on a stage and a named barrier
// hands its verdict to the other consumers (so they all stop together), and the producer's waits give up the same way
// (status word bit CSPB_DEV_TIMEOUT); before it returns after a failed wait the producer waits, bounded, for the
// copies it has issued.
#pragma once

#include "rowpass.cuh"
#include "mbar.cuh"

namespace cspb {

constexpr int kBulkThreads = kPassThreads + 32;  // 8 consumer warps + 1 producer warp
constexpr int kStageRows = 32;                   // 8 rows of each of the 4 warp rows (WX = 2)

// One bulk copy global -> this CTA's shared memory, completing on `bar` (16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}
__device__ __forceinline__ uint64_t evict_last_policy() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ void fence_proxy_async_global() { asm volatile("fence.proxy.async.global;" ::: "memory"); }

// Shared-memory layout of one stage: the 32 row segments, then the row vectors (4 × 32 floats: u1, u2, cyA, cyB of
// the stage's rows), then the column vectors (3 × CW floats: v1, v2, xv of the unit's chunk).
template <typename LT>
struct StageLayout {
    static constexpr int CW = PassGeo<LT, 2>::CW;
    static constexpr uint32_t row_bytes = uint32_t(CW) * sizeof(LT);  // 1024 for f32 and bf16
    static constexpr uint32_t data = kStageRows * row_bytes;
    static constexpr uint32_t rows_off = data;
    static constexpr uint32_t cols_off = rows_off + 4 * kStageRows * 4;
    static constexpr uint32_t bytes = cols_off + 3 * CW * 4;  // a multiple of 128
};

// The ring: NST stages, their barriers, the unit each stage belongs to (-1: the pass is over), the verdicts.
template <typename LT, int NST>
struct Ring {
    static constexpr uint32_t stage_bytes = StageLayout<LT>::bytes;
    static constexpr uint32_t red_off = NST * stage_bytes;
    static constexpr uint32_t bar_off = red_off + uint32_t(pass_smem_bytes<LT, 2>());
    static constexpr uint32_t total = bar_off + NST * 16 + NST * 4 + 16;
    unsigned char* base;
    __device__ unsigned char* stage(int i) const { return base + size_t(i) * stage_bytes; }
    __device__ unsigned char* red() const { return base + red_off; }
    __device__ uint64_t* full(int i) const { return reinterpret_cast<uint64_t*>(base + bar_off) + i; }
    __device__ uint64_t* empty(int i) const { return reinterpret_cast<uint64_t*>(base + bar_off) + NST + i; }
    __device__ int* unit_of(int i) const { return reinterpret_cast<int*>(base + bar_off + NST * 16) + i; }
    __device__ volatile int* verdict() const { return reinterpret_cast<volatile int*>(base + bar_off + NST * 20); }
    __device__ volatile int* abort_flag() const { return verdict() + 2; }
};

// What a pass reads per unit (flags as pass_unit's).
struct BulkPass {
    PassArgs a;
    bool rank2, csa, csb, rdot;
    bool reverse;   // walk the units from the last one (pass 2: recently written rows still in L2)
    int work_word;  // ctrl word of the pass's work counter
    int64_t units;
    uint64_t policy;  // L2 policy of the matrix copies
};

// Producer (warp 8): grabs units, issues their 4 stages, then one end-of-pass stage. q: the running stage count.
template <typename LT, int NST>
__device__ __forceinline__ bool bulk_produce(const Ring<LT, NST>& R, const BulkPass& P, uint32_t* ctrl, uint32_t& q) {
    using SL = StageLayout<LT>;
    constexpr int CW = SL::CW;
    const int lane = threadIdx.x & 31;
    const PassArgs& a = P.a;
    const int64_t n = a.n;
    for (;;) {
        int64_t unit = -1;
        if (lane == 0) {
            const uint32_t u = atomicAdd(ctrl + P.work_word, 1u);
            unit = u < P.units ? (P.reverse ? P.units - 1 - int64_t(u) : int64_t(u)) : -1;
        }
        unit = __shfl_sync(kFull, unit, 0);
        const int stages = unit < 0 ? 1 : 4;
        for (int s = 0; s < stages; ++s, ++q) {
            const int slot = int(q % NST);
            const uint32_t par = ((q / NST) & 1u) ^ 1u;
            int ok = 1;
            if (lane == 0) ok = mbar_wait(R.empty(slot), par, R.abort_flag(), ctrl) ? 1 : 0;
            ok = __shfl_sync(kFull, ok, 0);
            if (!ok) {
                *R.abort_flag() = 1;
                return false;
            }
            unsigned char* st = R.stage(slot);
            if (unit < 0) {
                if (lane == 0) {
                    *R.unit_of(slot) = -1;
                    mbar_arrive(R.full(slot));
                }
                __syncwarp();
                ++q;
                return true;
            }
            const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
            const int64_t r0 = strip * PassGeo<LT, 2>::S;
            const int64_t cbase = chunk * CW;
            const int64_t ccols = n - cbase < CW ? n - cbase : CW;  // a multiple of the vector width
            // rows of this stage per warp row wy: 8 unless the matrix ends inside the strip
            uint32_t total = 0;
#pragma unroll
            for (int wy = 0; wy < 4; ++wy) {
                const int64_t rr = n - (r0 + wy * 32 + 8 * s);
                const uint32_t rows = rr <= 0 ? 0u : (rr >= 8 ? 8u : uint32_t(rr));
                total += rows * uint32_t(ccols * sizeof(LT));
                const uint32_t vb = rows * 4u;
                total += vb * ((P.rank2 ? 2u : 0u) + (P.csa ? 1u : 0u) + (P.csb ? 1u : 0u));
            }
            if (s == 0) total += uint32_t(ccols) * 4u * ((P.rank2 ? 2u : 0u) + (P.rdot ? 1u : 0u));
            if (lane == 0) {
                *R.unit_of(slot) = int(unit);
                mbar_arrive_tx(R.full(slot), total);
            }
            __syncwarp();
            // lane L: row segment L (warp row L / 8, row 8s + L % 8 of it)
            {
                const int wy = lane >> 3, k = lane & 7;
                const int64_t row = r0 + wy * 32 + 8 * s + k;
                if (row < n)
                    bulk_g2s(st + size_t(lane) * SL::row_bytes, static_cast<const LT*>(a.src) + row * a.lds + cbase,
                             uint32_t(ccols * sizeof(LT)), R.full(slot), P.policy);
            }
            // lanes 0..15: row vectors (vector lane / 4, warp row lane % 4); lanes 16..18: column vectors
            if (lane < 16) {
                const int which = lane >> 2, wy = lane & 3;
                const float* v = which == 0 ? (P.rank2 ? a.u1 : nullptr)
                               : which == 1 ? (P.rank2 ? a.u2 : nullptr)
                               : which == 2 ? (P.csa ? a.cyA : nullptr)
                                            : (P.csb ? a.cyB : nullptr);
                const int64_t rr0 = r0 + wy * 32 + 8 * s;
                const int64_t rr = n - rr0;
                const uint32_t rows = rr <= 0 ? 0u : (rr >= 8 ? 8u : uint32_t(rr));
                if (v && rows)
                    bulk_g2s(st + SL::rows_off + (which * kStageRows + wy * 8) * 4, v + rr0, rows * 4u, R.full(slot),
                             0ull);
            } else if (lane < 19 && s == 0) {
                const int which = lane - 16;
                const float* v = which == 0 ? (P.rank2 ? a.v1 : nullptr)
                               : which == 1 ? (P.rank2 ? a.v2 : nullptr)
                                            : (P.rdot ? a.xv : nullptr);
                if (v) bulk_g2s(st + SL::cols_off + which * CW * 4, v + cbase, uint32_t(ccols) * 4u, R.full(slot), 0ull);
            }
        }
    }
}

// After a failed wait the producer waits (bounded) for every copy it issued that no consumer has seen complete.
template <typename LT, int NST>
__device__ __forceinline__ void bulk_drain(const Ring<LT, NST>& R, uint32_t q, uint32_t* ctrl) {
    if ((threadIdx.x & 31) != 0) return;
    const uint32_t from = q > uint32_t(NST) ? q - NST : 0u;
    for (uint32_t i = from; i < q; ++i) {
        const unsigned long long t0 = globaltimer_ns();
        while (!mbar_test(R.full(int(i % NST)), (i / NST) & 1u))
            if (globaltimer_ns() - t0 > kWaitBudgetNs) break;
    }
}

// Consumers (threads 0..255): one unit = 4 stages, the same arithmetic as pass_unit<LT, 2, ...>.
template <typename LT, int NST, bool RANK2, bool CSA, bool CSB, bool RDOT, bool DEFER = false>
__device__ __forceinline__ bool bulk_consume(const Ring<LT, NST>& R, const PassArgs& a, uint32_t* ctrl, uint32_t& q) {
    using G = PassGeo<LT, 2>;
    using SL = StageLayout<LT>;
    constexpr int VEC = G::VEC, CW = G::CW;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wx = warp % 2, wy = warp / 2;
    const int64_t n = a.n;
    const bool store = a.dst != nullptr;
    for (;;) {
        // the first stage of a unit (or the end of the pass)
        int slot = int(q % NST);
        if (threadIdx.x == 0) {
            const bool ok = mbar_wait(R.full(slot), (q / NST) & 1u, R.abort_flag(), ctrl);
            R.verdict()[q & 1] = ok ? 1 : 0;
            if (!ok) *R.abort_flag() = 1;
        }
        ConsumerSync{}();
        if (!R.verdict()[q & 1]) return false;
        const int unit_i = *R.unit_of(slot);
        if (unit_i < 0) {
            __syncwarp();
            if (lane == 0) mbar_arrive(R.empty(slot));
            ++q;
            return true;
        }
        const int64_t unit = unit_i;
        const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
        const int64_t r0 = strip * G::S + wy * 32;
        const int64_t c0 = chunk * CW + int64_t(wx * 32 + lane) * VEC;
        const int64_t rem_r = n - r0, rem_c = n - c0;
        const int nrows = rem_r <= 0 ? 0 : (rem_r >= 32 ? 32 : int(rem_r));
        const int ncols = rem_c <= 0 ? 0 : (rem_c >= VEC ? VEC : int(rem_c));
        double accA[VEC], accB[VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) { accA[e] = 0.0; accB[e] = 0.0; }
        float pA[VEC], pB[VEC];  // f32 partials of 8 rows (16-bit storage only)
#pragma unroll
        for (int e = 0; e < VEC; ++e) { pA[e] = 0.f; pB[e] = 0.f; }
        float racc[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) racc[k] = 0.f;
        float v1c[VEC], v2c[VEC], xc[VEC];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (s > 0) {
                slot = int(q % NST);
                if (threadIdx.x == 0) {
                    const bool ok = mbar_wait(R.full(slot), (q / NST) & 1u, R.abort_flag(), ctrl);
                    R.verdict()[q & 1] = ok ? 1 : 0;
                    if (!ok) *R.abort_flag() = 1;
                }
                ConsumerSync{}();
                if (!R.verdict()[q & 1]) return false;
            }
            const unsigned char* st = R.stage(slot);
            const float* rv = reinterpret_cast<const float*>(st + SL::rows_off);
            const float* cv = reinterpret_cast<const float*>(st + SL::cols_off);
            if (s == 0) {
#pragma unroll
                for (int e = 0; e < VEC; ++e) {
                    const bool ok = e < ncols;
                    const int cc = (wx * 32 + lane) * VEC + e;
                    v1c[e] = (RANK2 && ok) ? cv[cc] : 0.f;
                    v2c[e] = (RANK2 && ok) ? cv[CW + cc] : 0.f;
                    xc[e] = (RDOT && ok) ? cv[2 * CW + cc] : 0.f;
                }
            }
            const int kb = 8 * s;
            if (kb < nrows) {  // warp-uniform
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const int kk = kb + k;
                    const int sr = wy * 8 + k;  // the row's slot in the stage
                    if (kk < nrows) {
                        uint4 raw = make_uint4(0u, 0u, 0u, 0u);
                        if (ncols > 0)
                            raw = *reinterpret_cast<const uint4*>(st + size_t(sr) * SL::row_bytes +
                                                                  size_t((wx * 32 + lane) * VEC) * sizeof(LT));
                        const float u1k = RANK2 ? rv[sr] : 0.f;
                        const float u2k = RANK2 ? rv[kStageRows + sr] : 0.f;
                        const float cyak = CSA ? rv[2 * kStageRows + sr] : 0.f;
                        const float cybk = CSB ? rv[3 * kStageRows + sr] : 0.f;
                        float val[VEC];
                        unpack<LT>(raw, val);
                        float b[VEC];
#pragma unroll
                        for (int e = 0; e < VEC; ++e)
                            b[e] = RANK2 ? __fadd_rn(__fadd_rn(val[e], __fmul_rn(u1k, v1c[e])), __fmul_rn(u2k, v2c[e]))
                                         : val[e];
                        if (store && ncols > 0) store_vec<VEC>(a.dst + (r0 + kk) * a.ldd, c0, ncols, true, b);
                        if constexpr (kF32Part<LT>) {
                            // 16-bit storage: 8 products of a column in f32, then into the f64 sum (one conversion per 8 rows)
                            const bool flush = (kk & 7) == 7 || kk == nrows - 1;
                            if (CSA) {
#pragma unroll
                                for (int e = 0; e < VEC; ++e) pA[e] = fmaf(val[e], cyak, pA[e]);
                                if (flush) {
#pragma unroll
                                    for (int e = 0; e < VEC; ++e) { accA[e] += double(pA[e]); pA[e] = 0.f; }
                                }
                            }
                            if (CSB) {
#pragma unroll
                                for (int e = 0; e < VEC; ++e) pB[e] = fmaf(b[e], cybk, pB[e]);
                                if (flush) {
#pragma unroll
                                    for (int e = 0; e < VEC; ++e) { accB[e] += double(pB[e]); pB[e] = 0.f; }
                                }
                            }
                        } else {
                            if (CSA) {
#pragma unroll
                                for (int e = 0; e < VEC; ++e) accA[e] = __fma_rn(double(val[e]), double(cyak), accA[e]);
                            }
                            if (CSB) {
#pragma unroll
                                for (int e = 0; e < VEC; ++e) accB[e] = __fma_rn(double(b[e]), double(cybk), accB[e]);
                            }
                        }
                        if (RDOT) {
                            float d = 0.f;
#pragma unroll
                            for (int e = 0; e < VEC; ++e) d = fmaf(b[e], xc[e], d);
                            racc[kk] = d;
                        }
                    }
                }
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(R.empty(slot));
            ++q;
        }
        unit_epilogue<LT, 2, CSA, CSB, RDOT, ConsumerSync, DEFER>(a, strip, chunk, accA, accB, racc, R.red(),
                                                                  ConsumerSync{});
    }
}

}  // namespace cspb
