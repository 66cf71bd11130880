// gemver.cu — GEMVER, BiCGK and the gemver chain as persistent cooperative kernels built from rowpass.cuh.
//
// GEMVER, panel-pipelined (flag CSPB_GEMVER_PANEL; one launch, no grid barrier):
//   A column panel (CW columns × all n rows) is the unit of dependency: the row-dot partials of panel c need only
//   x over panel c, which needs only panel c's column sums. The work list runs pass 1 over panel c (read A, write Â,
//   f64 column partials of Â·y: Rank2Update + GemvTPartial fused), the block finishing the panel's last strip forms
//   x over the panel (ColReduce<true>, fixed order) and raises the panel's flag, and pass 2 over panel c (row dots
//   with x: Gemv) is scheduled one panel later, while the panel's Â (n·CW·4 bytes, 16 MB at n = 16384) is still in
//   L2. HBM traffic is then A once and Â once (8n² bytes in f32) instead of the 12n² of three streaming passes; the
//   last block to finish a strip's row partials writes w = α·dot. A pass-2 block waits (bounded) only on pass-1 work
//   already taken by running blocks, which never waits itself: no co-residency is assumed.
// GEMVER, three streaming passes (the default; cooperative launch). Measured faster than the panel schedule at
// n = 16384 on B200 although it moves a third more bytes: the panel order reads 1 KB row segments of ~2 panels at
// a time across every row, which HBM serves less efficiently than the strip order's whole rows.
//   pass 1   read A, write Â, f64 column partials        | grid barrier, x = z + β·Σ partials, grid barrier
//   pass 2   read Â (or A again), row dot partials with x, walked from the last strip back (recently written Â in
//            L2), 16 rows in flight per lane | grid barrier, w = α·Σ partials (rowsum_finish)
// Deferring the row sums to a phase of their own keeps the fence, the atomic and the last block's sums off every
// pass-2 unit (at n = 16384 pass 2 went from 4.3 to 5.5 TB/s); the sums run in the same order either way.
// flags = CSPB_GEMVER_BULK runs the same three passes with the matrix streamed through a shared-memory ring by bulk
// asynchronous copies (bulkpass.cuh). Measured at n = 16384 on B200 it is slower (0.87 vs 0.58 ms: pass 1 at
// 4.3 TB/s and pass 2 at 3.1 TB/s against 6.0 and 5.5): one CTA per SM leaves 8 consumer warps where the register
// pipeline runs 16, and the per-stage hand-off serialises them. It is kept as an option; results are the same bits.
// All schedules produce bit-identical results (the same partials, combined in the same order).
// BiCGK (one pass): q = B·p row dots and s = Bᵀ·r column partials from the same loads; one barrier; s.
// Chain (G1 → BiCGK → G2, six passes — the reference's nominal traffic counts eight), in two launches:
//   1: A0 → B1 + x1 partials | 2: B1 → w1 = α·(B1·x1), q = B1·x1 (p = x1, so one dot gives both)
//   3: B1 → s partials (with w1) + B2 + x2 partials (with q) | 4: B2 → w2.
#include <cstdio>
#include <initializer_list>

#include "bulkpass.cuh"

namespace cspb {

constexpr int kWX = 2;  // warps across columns in every GEMVER-family pass

struct GemverK {
    PassArgs p1, p2;
    uint32_t* ctrl;
    int64_t units;
    const float* z;
    float beta;
    float* x;
};

// The f32 row-dot passes over a stored Â (GEMVER's pass 2, the chain's passes 2 and 4, a row shard's finish) with the
// unit's cross-warp sums deferred as in lrd: each warp's 32 row dots go to one of two buffers, and the next unit forms Wp after its first loads. The
// arithmetic and its order are pass_unit<float, kWX, NC, false, false, false, true, 16, true>'s.
namespace p2f {

using G = PassGeo<float, kWX>;
constexpr int VEC = G::VEC, S = G::S, CW = G::CW, RB = 16;

__device__ __forceinline__ void rd_sum(const PassArgs& a, int64_t unit, const float* red2) {
    const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
    for (int t = threadIdx.x; t < S; t += kPassThreads) {
        const int64_t row = strip * S + t;
        if (row < a.rows) {
            float s = red2[t];
#pragma unroll
            for (int x = 1; x < kWX; ++x) s += red2[x * S + t];
            a.Wp[chunk * a.n + row] = s;
        }
    }
}

template <bool NC, class Pending>
__device__ __forceinline__ void unit(const PassArgs& a, int64_t unit, bool vec_ok, float* red_out, Pending&& pending) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wx = warp % kWX, wy = warp / kWX;
    const int64_t n = a.n;
    const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
    const int64_t r0 = strip * S + wy * 32;
    const int64_t c0 = chunk * CW + int64_t(wx * 32 + lane) * VEC;
    const int64_t rem_r = a.rows - r0, rem_c = n - c0;
    const int nrows = rem_r <= 0 ? 0 : (rem_r >= 32 ? 32 : int(rem_r));
    const int ncols = rem_c <= 0 ? 0 : (rem_c >= VEC ? VEC : int(rem_c));
    float xc[VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) xc[e] = e < ncols ? __ldcg(a.xv + c0 + e) : 0.f;
    float racc[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) racc[k] = 0.f;
    const float* src = static_cast<const float*>(a.src);
    const int64_t lds = a.lds;
#pragma unroll
    for (int kb = 0; kb < 32; kb += RB) {
        uint4 raw[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k)
            raw[k] = (kb + k < nrows && ncols > 0) ? load_raw<float, NC>(src + (r0 + kb + k) * lds, c0, ncols, vec_ok)
                                                   : make_uint4(0u, 0u, 0u, 0u);
        if (kb == 0) pending();
#pragma unroll
        for (int k = 0; k < RB; ++k) {
            const int kk = kb + k;
            if (kk < nrows) {
                float b[VEC];
                unpack<float>(raw[k], b);
                float d = 0.f;
#pragma unroll
                for (int e = 0; e < VEC; ++e) d = fmaf(b[e], xc[e], d);
                racc[kk] = d;
            }
        }
    }
    red_out[wx * S + wy * 32 + lane] = transpose_reduce32(racc);
}

// The pass over the units of counter `word`, from the last unit back (the rows written last are still in L2).
template <bool NC>
__device__ __forceinline__ void pass(const PassArgs& a, uint32_t* ctrl, int word, int64_t units, bool vec_ok) {
    __shared__ float rd[2][kWX * S];
    int64_t pend = -1;
    int slot = 0;
    for (uint32_t u = grab_work(ctrl, word); int64_t(u) < units;) {
        const uint32_t next = prefetch_work(ctrl, word);
        const int64_t cur = units - 1 - int64_t(u);
        unit<NC>(a, cur, vec_ok, rd[slot], [&] {
            if (pend >= 0) rd_sum(a, pend, rd[slot ^ 1]);
        });
        pend = cur;
        slot ^= 1;
        u = share_work(next);  // its barrier orders this unit's buffer stores before their sums
    }
    if (pend >= 0) rd_sum(a, pend, rd[slot ^ 1]);
}

}  // namespace p2f

template <typename T, bool P2_FROM_B>
__global__ void __launch_bounds__(kPassThreads, 2) k_gemver(GemverK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, kWX>()];
    for (uint32_t u = grab_work(g.ctrl, kWork0); u < g.units;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0);
        pass_unit<T, kWX, true, true, false, true, false, sizeof(T) == 4 ? 16 : 0>(g.p1, u, vec_ok != 0, smem);
        u = share_work(next);
    }
    if (!grid_barrier(g.ctrl)) return;
    colsum_finish(g.p1.PB, g.p1.strips, g.p1.n, g.z, g.beta, g.x);
    if (!grid_barrier(g.ctrl)) return;
    if constexpr (P2_FROM_B) {
        p2f::pass<false>(g.p2, g.ctrl, kWork0 + 1, g.units, vec_ok != 0);
    } else {
        for (uint32_t u = grab_work(g.ctrl, kWork0 + 1); u < g.units;) {
            const uint32_t next = prefetch_work(g.ctrl, kWork0 + 1);
            pass_unit<T, kWX, true, true, false, false, true, 0, true>(g.p2, g.units - 1 - int64_t(u), vec_ok != 0,
                                                                       smem);
            u = share_work(next);
        }
    }
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish(g.p2);
}

// GEMVER without Â (flag CSPB_GEMVER_LOWRANK, B not requested): the rank-2 update is applied as four dot products,
//   Âᵀy = Aᵀy + v1(u1·y) + v2(u2·y),   Â·x = A·x + u1(v1·x) + u2(v2·x),
// so the two passes over A are plain streaming GEMVs (column sums of A·y, then row dots of A·x) with no per-element
// update, and the finishes add the rank-2 terms. The dots are formed in f64 by block 0 (block_dot2, one fixed order)
// and handed to every block through the control block. Measured at n = 16384 with bf16 storage, forming Â per element made each pass issue-bound at 3.3 TB/s.
// Other rounding than the schedules that form Â (closer to the f64 result, not the same bits).
struct LowRankK {
    PassArgs p1, p2;
    uint32_t* ctrl;
    int64_t units;
    const float *u1, *v1, *u2, *v2, *y, *z;
    float beta;
    float* x;
};

// STORE: Â is requested (16-bit A only): pass 1 forms and stores it and x comes from its column sums, as k_gemver's;
// only pass 2 takes the low-rank form (w from A, the rank-2 terms in the finish) instead of forming Â again.
// 16-bit A without Â: rows per load batch and blocks per SM of the two streaming passes (8 rows, 3 blocks: 24 warps per
// SM with 128 B per lane in flight)
template <typename T, bool STORE> inline constexpr int kLrRB = (sizeof(T) == 2 && !STORE) ? 8 : 16;
template <typename T, bool STORE> inline constexpr int kLrBlocks = (sizeof(T) == 2 && !STORE) ? 3 : 2;

// ---- the bf16 low-rank passes with the unit's cross-warp sums deferred ------------------------------------------------
// pass_unit ends each unit with two block barriers: the warps of a unit store their column sums (pass 1) or row dots
// (pass 2) to shared memory, wait for one another, and sum across warps. Here each warp stores its share into one of
// two buffers and goes on; the next unit's threads form those sums right after issuing their first loads (the
// barrier of the work hand-off between the units orders the stores before them), so the sums overlap the loads in
// flight and the unit has no barrier of its own. The arithmetic and its order are pass_unit's
// (<bf16, kWX, NC, !RANK2, !CSA, CSB | RDOT, RB, DEFER>), so the results are the same bits, as the task runner's.
namespace lrd {

using Bf = __nv_bfloat16;
using G = PassGeo<Bf, kWX>;
constexpr int VEC = G::VEC, WY = G::WY, S = G::S, CW = G::CW;

// The two passes run apart (grid barriers between them), so their buffers share the block's shared memory.
union Bufs {
    double cs[2][WY * CW];  // pass 1: each warp's column sums, two units' worth
    struct {
        float rd[2][kWX * S];                    // each warp's row dots, two units' worth
        float rdot[kPassThreads / 32][32 * 32];  // a warp's dots of its 32 rows, [row][lane]
    } p2;
};

// pass 1's sums of unit `unit` from buffer `slot`: P[strip][col] = ((w0 + w1) + w2) + w3 over the row warps
__device__ __forceinline__ void cs_sum(const PassArgs& a, int64_t unit, const double* red) {
    const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
    for (int t = threadIdx.x; t < CW; t += kPassThreads) {
        const int64_t col = chunk * CW + t;
        if (col < a.n) {
            double s = red[t];
#pragma unroll
            for (int y = 1; y < WY; ++y) s += red[y * CW + t];
            a.PB[strip * a.n + col] = s;
        }
    }
}
// pass 2's row dots of unit `unit`: Wp[chunk][row] = w0 + w1 over the column warps
__device__ __forceinline__ void rd_sum(const PassArgs& a, int64_t unit, const float* red2) {
    const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
    for (int t = threadIdx.x; t < S; t += kPassThreads) {
        const int64_t row = strip * S + t;
        if (row < a.rows) {
            float s = red2[t];
#pragma unroll
            for (int x = 1; x < kWX; ++x) s += red2[x * S + t];
            a.Wp[chunk * a.n + row] = s;
        }
    }
}

// One unit; `pending` runs once, after the first batch's loads are issued (the previous unit's sums).
template <bool CS, int RB, class Pending>
__device__ __forceinline__ void unit(const PassArgs& a, int64_t unit, bool vec_ok, Bufs& B, int slot,
                                     Pending&& pending) {
    static_assert(32 % RB == 0, "batches of rows that divide the warp's 32");
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wx = warp % kWX, wy = warp / kWX;
    const int64_t n = a.n;
    const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
    const int64_t r0 = strip * S + wy * 32;
    const int64_t c0 = chunk * CW + int64_t(wx * 32 + lane) * VEC;
    const int64_t rem_r = a.rows - r0, rem_c = n - c0;
    const int nrows = rem_r <= 0 ? 0 : (rem_r >= 32 ? 32 : int(rem_r));
    const int ncols = rem_c <= 0 ? 0 : (rem_c >= VEC ? VEC : int(rem_c));
    float cybr = 0.f;
    if (CS && lane < nrows) cybr = __ldcg(a.cyB + r0 + lane);
    float xc[VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) xc[e] = (!CS && e < ncols) ? __ldcg(a.xv + c0 + e) : 0.f;
    double accB[VEC];
    float pB[VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) { accB[e] = 0.0; pB[e] = 0.f; }
    const Bf* src = static_cast<const Bf*>(a.src);
    const int64_t lds = a.lds;
    float* rdot = B.p2.rdot[warp];
#pragma unroll 1
    for (int kb = 0; kb < 32; kb += RB) {
        uint4 raw[RB];
#pragma unroll
        for (int k = 0; k < RB; ++k)
            raw[k] = (kb + k < nrows && ncols > 0) ? load_raw<Bf, true>(src + (r0 + kb + k) * lds, c0, ncols, vec_ok)
                                                   : make_uint4(0u, 0u, 0u, 0u);
        if (kb == 0) pending();
        if (kb < nrows) {
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                const int kk = kb + k;
                const float cybk = __shfl_sync(kFull, cybr, kk);
                if (kk < nrows) {
                    float b[VEC];
                    unpack<Bf>(raw[k], b);
                    if constexpr (CS) {
                        const bool flush = (kk & 7) == 7 || kk == nrows - 1;
#pragma unroll
                        for (int e = 0; e < VEC; ++e) pB[e] = fmaf(b[e], cybk, pB[e]);
                        if (flush) {
#pragma unroll
                            for (int e = 0; e < VEC; ++e) { accB[e] += double(pB[e]); pB[e] = 0.f; }
                        }
                    } else {
                        float d = 0.f;
#pragma unroll
                        for (int e = 0; e < VEC; ++e) d = fmaf(b[e], xc[e], d);
                        rdot[kk * 32 + lane] = d;
                    }
                }
            }
        }
    }
    if constexpr (CS) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) B.cs[slot][wy * CW + (wx * 32 + lane) * VEC + e] = accB[e];
    } else {
        float racc[32];
#pragma unroll
        for (int k = 0; k < 32; ++k) racc[k] = k < nrows ? rdot[k * 32 + lane] : 0.f;  // this lane's own values
        B.p2.rd[slot][wx * S + wy * 32 + lane] = transpose_reduce32(racc);
    }
}

}  // namespace lrd

template <typename T, bool STORE>
__global__ void __launch_bounds__(kPassThreads, (kLrBlocks<T, STORE>)) k_gemver_lr(LowRankK g, int vec_ok) {
    constexpr int RB = kLrRB<T, STORE>;
    // pass 1's pass_unit and pass 2's deferred sums run apart (grid barriers between them): one block of shared memory
    __shared__ union {
        __align__(16) unsigned char smem[pass_smem_bytes<T, kWX>()];
        lrd::Bufs B;
    } sh;
    unsigned char* smem = sh.smem;
    // The dot products of the finishes are formed by block 0 alone (block_dot2: one order, whatever the grid) and read
    // by every block after the next grid barrier; every block forming them read 3 vectors each time (85 MB of L2 reads
    // per finish at n = 16384 and 444 blocks).
    double* dots = reinterpret_cast<double*>(g.ctrl + kDots0);
    if constexpr (!STORE) {
        if (blockIdx.x == 0) {  // u1·y, u2·y: inputs only
            double s1, s2;
            block_dot2(g.u1, g.u2, g.y, g.p1.n, s1, s2);
            if (threadIdx.x == 0) {
                dots[0] = s1;
                dots[1] = s2;
            }
        }
    }
    for (uint32_t u = grab_work(g.ctrl, kWork0); u < g.units;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0);
        if constexpr (STORE) pass_unit<T, kWX, true, true, false, true, false, 0>(g.p1, u, vec_ok != 0, smem);
        else pass_unit<T, kWX, true, false, false, true, false, RB>(g.p1, u, vec_ok != 0, smem);
        u = share_work(next);
    }
    if (!grid_barrier(g.ctrl)) return;
    if constexpr (STORE) {
        colsum_finish(g.p1.PB, g.p1.strips, g.p1.n, g.z, g.beta, g.x);
    } else {
        colsum_finish_lr(g.p1.PB, g.p1.strips, g.p1.n, g.z, g.beta, g.v1, g.v2, __ldcg(dots), __ldcg(dots + 1), g.x);
    }
    if (!grid_barrier(g.ctrl)) return;
    if (blockIdx.x == 0) {  // v1·x, v2·x: x is complete after the barrier
        double t1, t2;
        block_dot2(g.v1, g.v2, g.x, g.p2.n, t1, t2);
        if (threadIdx.x == 0) {
            dots[2] = t1;
            dots[3] = t2;
        }
    }
    // pass 2 with the cross-warp sums of each unit deferred to the next unit (the same bits as pass_unit's)
    if constexpr (sizeof(T) == 4) {
        p2f::pass<true>(g.p2, g.ctrl, kWork0 + 1, g.units, vec_ok != 0);
    } else {
        int64_t pend = -1;
        int slot = 0;
        for (uint32_t u = grab_work(g.ctrl, kWork0 + 1); u < g.units;) {
            const uint32_t next = prefetch_work(g.ctrl, kWork0 + 1);
            const int64_t cur = g.units - 1 - int64_t(u);
            lrd::unit<false, RB>(g.p2, cur, vec_ok != 0, sh.B, slot, [&] {
                if (pend >= 0) lrd::rd_sum(g.p2, pend, sh.B.p2.rd[slot ^ 1]);
            });
            pend = cur;
            slot ^= 1;
            u = share_work(next);
        }
        if (pend >= 0) lrd::rd_sum(g.p2, pend, sh.B.p2.rd[slot ^ 1]);
    }
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish_lr(g.p2, g.u1, g.u2, __ldcg(dots + 2), __ldcg(dots + 3));
}



// k_gemver_lr<bf16, false> with the deferred cross-warp sums (lrd::unit): the same bits, no barrier inside a unit.
__global__ void __launch_bounds__(kPassThreads, (kLrBlocks<__nv_bfloat16, false>)) k_gemver_lr_bf16(LowRankK g,
                                                                                                    int vec_ok) {
    constexpr int RB = kLrRB<__nv_bfloat16, false>;
    __shared__ lrd::Bufs B;
    double* dots = reinterpret_cast<double*>(g.ctrl + kDots0);
    if (blockIdx.x == 0) {  // u1·y, u2·y: inputs only
        double s1, s2;
        block_dot2(g.u1, g.u2, g.y, g.p1.n, s1, s2);
        if (threadIdx.x == 0) {
            dots[0] = s1;
            dots[1] = s2;
        }
    }
    {
        int64_t pend = -1;
        int slot = 0;
        for (uint32_t u = grab_work(g.ctrl, kWork0); u < g.units;) {
            const uint32_t next = prefetch_work(g.ctrl, kWork0);
            lrd::unit<true, RB>(g.p1, u, vec_ok != 0, B, slot, [&] {
                if (pend >= 0) lrd::cs_sum(g.p1, pend, B.cs[slot ^ 1]);
            });
            pend = u;
            slot ^= 1;
            u = share_work(next);  // its barrier orders this unit's buffer stores before their sums
        }
        if (pend >= 0) lrd::cs_sum(g.p1, pend, B.cs[slot ^ 1]);
    }
    if (!grid_barrier(g.ctrl)) return;
    colsum_finish_lr(g.p1.PB, g.p1.strips, g.p1.n, g.z, g.beta, g.v1, g.v2, __ldcg(dots), __ldcg(dots + 1), g.x);
    if (!grid_barrier(g.ctrl)) return;
    if (blockIdx.x == 0) {  // v1·x, v2·x: x is complete after the barrier
        double t1, t2;
        block_dot2(g.v1, g.v2, g.x, g.p2.n, t1, t2);
        if (threadIdx.x == 0) {
            dots[2] = t1;
            dots[3] = t2;
        }
    }
    {
        int64_t pend = -1;
        int slot = 0;
        for (uint32_t u = grab_work(g.ctrl, kWork0 + 1); u < g.units;) {
            const uint32_t next = prefetch_work(g.ctrl, kWork0 + 1);
            lrd::unit<false, RB>(g.p2, g.units - 1 - int64_t(u), vec_ok != 0, B, slot, [&] {
                if (pend >= 0) lrd::rd_sum(g.p2, pend, B.p2.rd[slot ^ 1]);
            });
            pend = g.units - 1 - int64_t(u);
            slot ^= 1;
            u = share_work(next);
        }
        if (pend >= 0) lrd::rd_sum(g.p2, pend, B.p2.rd[slot ^ 1]);
    }
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish_lr(g.p2, g.u1, g.u2, __ldcg(dots + 2), __ldcg(dots + 3));
}

// The same three passes with the matrix streamed through a shared-memory ring by bulk copies (bulkpass.cuh): one
// CTA per SM, 8 consumer warps and a producer warp; the results are bit-identical to k_gemver's.
template <typename T, bool P2_FROM_B, int NST>
__global__ void __launch_bounds__(kBulkThreads, 1) k_gemver_bulk(GemverK g) {
    extern __shared__ __align__(128) unsigned char dsm[];
    const Ring<T, NST> R{dsm};
    const int warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; ++i) {
            mbar_init(R.full(i), 1);
            mbar_init(R.empty(i), kPassThreads / 32);
        }
        R.verdict()[0] = 0;
        R.verdict()[1] = 0;
        *R.abort_flag() = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    uint32_t q = 0;
    const uint64_t first = evict_first_policy();
    {
        BulkPass P{g.p1, true, false, true, false, false, kWork0, g.units, first};
        if (warp == kPassThreads / 32) {
            if (!bulk_produce<T, NST>(R, P, g.ctrl, q)) bulk_drain<T, NST>(R, q, g.ctrl);
        } else {
            bulk_consume<T, NST, true, false, true, false>(R, g.p1, g.ctrl, q);
        }
    }
    // pass 1's Â stores and the x of the finish are read by pass 2's bulk copies (the async proxy) in other CTAs
    fence_proxy_async_global();
    if (!grid_barrier(g.ctrl)) return;
    colsum_finish(g.p1.PB, g.p1.strips, g.p1.n, g.z, g.beta, g.x);
    fence_proxy_async_global();
    if (!grid_barrier(g.ctrl)) return;
    fence_proxy_async_global();
    {
        BulkPass P{g.p2, !P2_FROM_B, false, false, true, true, kWork0 + 1, g.units, first};
        if (warp == kPassThreads / 32) {
            if (!bulk_produce<T, NST>(R, P, g.ctrl, q)) bulk_drain<T, NST>(R, q, g.ctrl);
        } else {
            bulk_consume<T, NST, !P2_FROM_B, false, false, true, true>(R, g.p2, g.ctrl, q);
        }
    }
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish(g.p2);
}

struct PanelK {
    PassArgs p1, p2;
    uint32_t* ctrl;
    uint32_t* chunk_done;  // [chunks]
    uint32_t* x_ready;     // [chunks]
    const float* z;
    float beta;
    float* x;
    int64_t lag;           // pass 2 over panel c follows pass 1 over panel c + lag
};

// Block b of the work list (each block = one panel's strips) -> (pass, panel).
__device__ __forceinline__ void panel_block(int64_t b, int64_t C, int64_t L, int& pass, int64_t& c) {
    if (b < L) { pass = 1; c = b; return; }
    const int64_t r = b - L;
    if (r < 2 * (C - L)) {
        const int64_t t = L + r / 2;
        if ((r & 1) == 0) { pass = 1; c = t; }
        else { pass = 2; c = t - L; }
        return;
    }
    pass = 2;
    c = C - L + (r - 2 * (C - L));
}

template <typename T, bool P2_FROM_B>
__global__ void __launch_bounds__(kPassThreads, 2) k_gemver_panel(PanelK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, kWX>()];
    __shared__ int s_flag;
    const int64_t S = g.p1.strips, C = g.p1.chunks, L = g.lag;
    const int64_t items = 2 * S * C;
    constexpr int CW = PassGeo<T, kWX>::CW;
    for (;;) {
        const uint32_t item = grab_work(g.ctrl, kWork0);
        if (int64_t(item) >= items) break;
        int pass;
        int64_t c;
        panel_block(int64_t(item) / S, C, L, pass, c);
        const int64_t si = int64_t(item) % S;
        if (pass == 1) {
            pass_unit<T, kWX, true, true, false, true, false>(g.p1, si * C + c, vec_ok != 0, smem);
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) s_flag = atomicAdd(g.chunk_done + c, 1u) == uint32_t(S - 1);
            __syncthreads();
            if (s_flag) {  // the panel's last strip: x over the panel
                __threadfence();
                const int64_t c0 = c * CW, c1 = min(g.p1.n, c0 + CW);
                colsum_finish_cols(g.p1.PB, S, g.p1.n, c0, c1, g.z, g.beta, g.x);
                __threadfence();
                __syncthreads();
                if (threadIdx.x == 0) st_release(g.x_ready + c, 1u);
            }
        } else {
            if (threadIdx.x == 0) s_flag = ld_acquire(g.x_ready + c) != 0u || wait_change(g.x_ready + c, 0u, g.ctrl);
            __syncthreads();
            if (!s_flag) break;
            const int64_t unit = (S - 1 - si) * C + c;  // the panel's strips from the last one back
            if constexpr (P2_FROM_B)
                pass_unit<float, kWX, false, false, false, false, true>(g.p2, unit, vec_ok != 0, smem);
            else
                pass_unit<T, kWX, true, true, false, false, true>(g.p2, unit, vec_ok != 0, smem);
        }
    }
}

struct BicgkK {
    PassArgs p;
    uint32_t* ctrl;
    int64_t units;
    float* s;
};

template <typename T>
__global__ void __launch_bounds__(kPassThreads, 2) k_bicgk(BicgkK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, kWX>()];
    for (uint32_t u = grab_work(g.ctrl, kWork0); u < g.units;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0);
        pass_unit<T, kWX, true, false, false, true, true, sizeof(T) == 4 ? 16 : 0, true>(g.p, u, vec_ok != 0, smem);
        u = share_work(next);
    }
    if (!grid_barrier(g.ctrl)) return;
    colsum_finish(g.p.PB, g.p.strips, g.p.n, nullptr, 1.0f, g.s);
    rowsum_finish(g.p);
}

struct ChainK {
    PassArgs p1, p2, p3, p4;
    uint32_t* ctrl;
    int64_t units;
    const float* za;
    float beta;
    float *x1, *s, *x2;
};

// The chain runs as two cooperative launches: G1's passes (1, 2) and then BiCGK + G2's (3, 4). One fused launch
// measured slower at n = 16384 (1.41 vs 1.17 ms): with all four passes in one kernel the row-dot passes ran at
// 4.0 TB/s instead of 5.1, and the launch boundary is what lets pass 3 read B1 through the non-coherent path.
// First launch: 1: A0 -> B1, partials of B1ᵀ·ya | x1 | 2: B1 · x1 -> w1 (α) and q (1), from the last strip back.
__global__ void __launch_bounds__(kPassThreads, 2) k_chain_g1(ChainK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<float, kWX>()];
    const bool vo = vec_ok != 0;
    for (uint32_t u = grab_work(g.ctrl, kWork0); u < g.units;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0);
        pass_unit<float, kWX, true, true, false, true, false, 16>(g.p1, u, vo, smem);
        u = share_work(next);
    }
    if (!grid_barrier(g.ctrl)) return;
    colsum_finish(g.p1.PB, g.p1.strips, g.p1.n, g.za, g.beta, g.x1);
    if (!grid_barrier(g.ctrl)) return;
    p2f::pass<false>(g.p2, g.ctrl, kWork0 + 1, g.units, vo);
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish(g.p2);
}

// Second launch: 3: B1 -> partials of B1ᵀ·w1 (s); B2 = B1 + update; partials of B2ᵀ·q (x2) | s, x2 |
// 4: B2 · x2 -> w2, from the last strip back. B1_NC: B1 is read-only in this launch (B2 does not overlap it), so
// pass 3 streams it through the non-coherent path with evict-first, and L2 keeps the B2 rows pass 3 wrote last for
// pass 4 (measured: pass 3 at 6.3 TB/s instead of 4.6, pass 4 at 5.0 instead of 4.0).
template <bool B1_NC>
__global__ void __launch_bounds__(kPassThreads, 2) k_chain_g2(ChainK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<float, kWX>()];
    const bool vo = vec_ok != 0;
    for (uint32_t u = grab_work(g.ctrl, kWork0 + 2); u < g.units;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0 + 2);
        pass_unit<float, kWX, B1_NC, true, true, true, false, 16>(g.p3, u, vo, smem);
        u = share_work(next);
    }
    if (!grid_barrier(g.ctrl)) return;
    colsum_finish(g.p3.PA, g.p3.strips, g.p3.n, nullptr, 1.0f, g.s);    // s = B1ᵀ·w1
    colsum_finish(g.p3.PB, g.p3.strips, g.p3.n, g.s, g.beta, g.x2);     // x2 = s + β·B2ᵀ·q (same thread owns s[j])
    if (!grid_barrier(g.ctrl)) return;
    p2f::pass<false>(g.p4, g.ctrl, kWork0 + 3, g.units, vo);
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish(g.p4);
}

// Row shards of ONE GEMVER across GPUs (one process per GPU). A shard holds rows [r0, r0 + rows) of A, u1, u2, y and
// all of v1, v2, z. The only exchange is the column sums: Âᵀy = Σ over shards of the shard's rows' share.
//   partial: Â rows (stored when B is given) and the shard's f64 column sums colsum[j] = Σ_{i in shard} Â[i][j]·y[i]
//   (the caller adds the shards' colsum in rank order, the same total on every rank)
//   finish:  x = float(z + β·total) over all n columns, then w = α·Â·x over the shard's rows (pass 2 of k_gemver)
struct RowsK {
    PassArgs p;
    uint32_t* ctrl;
    int64_t units;
    double* colsum;
    const double* total;
    const float* z;
    float beta;
    float* x;
};

template <typename T>
__global__ void __launch_bounds__(kPassThreads, 2) k_rows_partial(RowsK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, kWX>()];
    for (uint32_t u = grab_work(g.ctrl, kWork0); u < g.units;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0);
        pass_unit<T, kWX, true, true, false, true, false, sizeof(T) == 4 ? 16 : 0>(g.p, u, vec_ok != 0, smem);
        u = share_work(next);
    }
    if (!grid_barrier(g.ctrl)) return;
    colsum_f64(g.p.PB, g.p.strips, g.p.n, g.colsum);
}

// FROM_B: the shard's Â rows were stored by the partial launch and are read-only here (the non-coherent path);
// otherwise A again, re-applying the update (as k_gemver's pass 2).
template <typename T, bool FROM_B>
__global__ void __launch_bounds__(kPassThreads, 2) k_rows_finish(RowsK g, int vec_ok) {
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, kWX>()];
    const int64_t n = g.p.n;
    const int64_t gthreads = int64_t(gridDim.x) * blockDim.x;
    for (int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += gthreads) {
        const double zz = g.z ? double(__ldcg(g.z + j)) : 0.0;
        g.x[j] = float(zz + double(g.beta) * __ldcg(g.total + j));
    }
    if (!grid_barrier(g.ctrl)) return;
    if constexpr (FROM_B) {
        p2f::pass<true>(g.p, g.ctrl, kWork0 + 1, g.units, vec_ok != 0);
    } else {
        for (uint32_t u = grab_work(g.ctrl, kWork0 + 1); u < g.units;) {
            const uint32_t next = prefetch_work(g.ctrl, kWork0 + 1);
            pass_unit<T, kWX, true, true, false, false, true, 0, true>(g.p, g.units - 1 - int64_t(u), vec_ok != 0,
                                                                       smem);
            u = share_work(next);
        }
    }
    if (!grid_barrier(g.ctrl)) return;
    rowsum_finish(g.p);
}

}  // namespace cspb

// =====================================================================================================================
// host side
// =====================================================================================================================
using namespace cspb;
using cspb_host::align_up;
using cspb_host::aligned;

namespace {

struct PassLayout {
    int64_t strips = 0, chunks = 0, units = 0;
    size_t off_done = 0, off_chunk = 0, off_PA = 0, off_PB = 0, off_Wp = 0, total = 0;
};

// Workspace: [ctrl 256][strip_done: strips u32 × nsets][chunk_done, x_ready: chunks u32 each]
//            [PA: strips×n f64][PB: strips×n f64][Wp: chunks×n f32]
// Everything before PA is zeroed per call.
PassLayout pass_layout(int64_t n, int S, int CW, int done_sets, bool want_PA) {
    PassLayout L;
    L.strips = (n + S - 1) / S;
    L.chunks = (n + CW - 1) / CW;
    L.units = L.strips * L.chunks;
    size_t o = kCtrlBytes;
    L.off_done = o;
    o = o + size_t(L.strips) * sizeof(uint32_t) * size_t(done_sets);
    L.off_chunk = o;
    o = align_up(o + 2 * size_t(L.chunks) * sizeof(uint32_t), 256);
    L.off_PA = o;
    if (want_PA) o = align_up(o + size_t(L.strips) * size_t(n) * sizeof(double), 256);
    L.off_PB = o;
    o = align_up(o + size_t(L.strips) * size_t(n) * sizeof(double), 256);
    L.off_Wp = o;
    o = align_up(o + size_t(L.chunks) * size_t(n) * sizeof(float), 256);
    L.total = o;
    return L;
}

constexpr int kS = PassGeo<float, kWX>::S;
constexpr int kCW32 = PassGeo<float, kWX>::CW;
constexpr int kCW16 = PassGeo<__nv_bfloat16, kWX>::CW;

template <typename K>
int launch_coop(K kernel, void** args, int64_t units, size_t zero_bytes, void* ws, cudaStream_t st) {
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    if (!di.coop) return CSPB_ERR_UNSUPPORTED;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPassThreads, 0);
    if (e != cudaSuccess || per_sm < 1) return e != cudaSuccess ? cspb_host::map_cuda_error(e) : CSPB_ERR_LAUNCH;
    int64_t grid = int64_t(per_sm) * di.sms;
    if (grid > units) grid = units;
    if (grid < 1) grid = 1;
    if (zero_bytes) {
        e = cudaMemsetAsync(ws, 0, zero_bytes, st);
        if (e != cudaSuccess) return cspb_host::map_cuda_error(e);
    }
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(unsigned(grid)), dim3(kPassThreads),
                                    args, 0, st);
    if (e != cudaSuccess) return CSPB_ERR_LAUNCH;
    return CSPB_OK;
}

template <typename K>
int launch_persistent(K kernel, void** args, int64_t items, size_t zero_bytes, void* ws, cudaStream_t st) {
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPassThreads, 0);
    if (e != cudaSuccess || per_sm < 1) return e != cudaSuccess ? cspb_host::map_cuda_error(e) : CSPB_ERR_LAUNCH;
    int64_t grid = int64_t(per_sm) * di.sms;
    if (grid > items) grid = items;
    if (grid < 1) grid = 1;
    e = cudaMemsetAsync(ws, 0, zero_bytes, st);
    if (e != cudaSuccess) return cspb_host::map_cuda_error(e);
    e = cudaLaunchKernel(reinterpret_cast<const void*>(kernel), dim3(unsigned(grid)), dim3(kPassThreads), args, 0, st);
    return e == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

template <typename K>
int launch_coop_bulk(K kernel, void** args, size_t smem, size_t zero_bytes, void* ws, cudaStream_t st) {
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    if (!di.coop) return CSPB_ERR_UNSUPPORTED;
    cudaError_t e = cudaFuncSetAttribute(reinterpret_cast<const void*>(kernel),
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
    if (e != cudaSuccess) return cspb_host::map_cuda_error(e);
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBulkThreads, smem);
    if (e != cudaSuccess || per_sm < 1) return e != cudaSuccess ? cspb_host::map_cuda_error(e) : CSPB_ERR_LAUNCH;
    const int64_t grid = int64_t(per_sm) * di.sms;
    if (zero_bytes) {
        e = cudaMemsetAsync(ws, 0, zero_bytes, st);
        if (e != cudaSuccess) return cspb_host::map_cuda_error(e);
    }
    e = cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kernel), dim3(unsigned(grid)), dim3(kBulkThreads),
                                    args, smem, st);
    return e == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

bool aligned16(std::initializer_list<const void*> ps) {
    for (const void* p : ps)
        if (p && !aligned(p, 16)) return false;
    return true;
}

bool vec_aligned(const void* p, int64_t ld, int elem_bytes) {
    return p == nullptr || (aligned(p, 16) && (ld * elem_bytes) % 16 == 0);
}

}  // namespace

extern "C" {

size_t cspb_gemver_workspace_bytes(int64_t n) {
    if (n < 1) return 0;
    return pass_layout(n, kS, kCW32, 1, false).total;  // the f32 layout has the most chunks
}

int cspb_gemver_fused(const cspb_gemver_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    const int64_t n = d->n;
    if (n < 1 || d->lda < n || (d->B && d->ldb < n)) return CSPB_ERR_ARGUMENT;
    if (n > (int64_t(1) << 31)) return CSPB_ERR_ARGUMENT;
    if (!d->A || !d->u1 || !d->v1 || !d->u2 || !d->v2 || !d->y || !d->x || !d->w) return CSPB_ERR_ARGUMENT;
    if (d->a_dtype != CSPB_F32 && d->a_dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    if ((d->flags & ~(CSPB_GEMVER_PANEL | CSPB_GEMVER_BULK | CSPB_GEMVER_LOWRANK | CSPB_GEMVER_LAG_MASK)) != 0)
        return CSPB_ERR_UNSUPPORTED;
    const bool bf16 = d->a_dtype == CSPB_BF16;
    const PassLayout L = pass_layout(n, kS, bf16 ? kCW16 : kCW32, 1, false);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    if (2 * L.units >= int64_t(0xffffffffll)) return CSPB_ERR_ARGUMENT;
    char* ws = static_cast<char*>(d->workspace);

    PassArgs p1{};
    p1.n = n;
    p1.rows = n;
    p1.src = d->A;
    p1.lds = d->lda;
    p1.dst = d->B;
    p1.ldd = d->ldb;
    p1.u1 = d->u1; p1.v1 = d->v1; p1.u2 = d->u2; p1.v2 = d->v2;
    p1.cyB = d->y;
    p1.PB = reinterpret_cast<double*>(ws + L.off_PB);
    p1.strips = L.strips;
    p1.chunks = L.chunks;
    PassArgs p2 = p1;
    p2.dst = nullptr;
    p2.cyB = nullptr;
    p2.PB = nullptr;
    p2.xv = d->x;
    p2.Wp = reinterpret_cast<float*>(ws + L.off_Wp);
    p2.strip_done = reinterpret_cast<uint32_t*>(ws + L.off_done);
    p2.rout1 = d->w;
    p2.rscale1 = d->alpha;
    const bool from_B = !bf16 && d->B != nullptr;
    if (from_B) {
        p2.src = d->B;
        p2.lds = d->ldb;
    }
    const int eb = bf16 ? 2 : 4;
    const int vec_ok = vec_aligned(d->A, d->lda, eb) && vec_aligned(d->B, d->ldb, 4) ? 1 : 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t zero = L.off_PA;  // ctrl, strip_done, chunk_done, x_ready

    // the low-rank form: without Â (any dtype), or with Â and a 16-bit matrix (pass 2 only); it takes precedence over
    // the schedule flags. With Â and an f32 matrix pass 2 reads the stored Â, and the flag is ignored.
    if ((d->flags & CSPB_GEMVER_LOWRANK) && (d->B == nullptr || bf16)) {
        const bool store = d->B != nullptr;
        LowRankK g{};
        g.p1 = p1;
        if (!store) {
            g.p1.dst = nullptr;
            g.p1.u1 = g.p1.v1 = g.p1.u2 = g.p1.v2 = nullptr;
        }
        g.p2 = p2;
        g.p2.src = d->A;  // pass 2 reads A (the 16-bit matrix), never the stored Â
        g.p2.lds = d->lda;
        g.ctrl = reinterpret_cast<uint32_t*>(ws);
        g.units = L.units;
        g.u1 = d->u1; g.v1 = d->v1; g.u2 = d->u2; g.v2 = d->v2;
        g.y = d->y;
        g.z = d->z;
        g.beta = d->beta;
        g.x = d->x;
        void* args[] = {&g, const_cast<int*>(&vec_ok)};
        if (bf16 && store) return launch_coop(k_gemver_lr<__nv_bfloat16, true>, args, L.units, zero, ws, st);
        if (bf16) return launch_coop(k_gemver_lr_bf16, args, L.units, zero, ws, st);
        return launch_coop(k_gemver_lr<float, false>, args, L.units, zero, ws, st);
    }
    // the bulk-copy ring: every row segment and vector piece must start on 16 bytes and be a multiple of 16 bytes long
    const int vw = bf16 ? 8 : 4;
    const bool bulk_ok = vec_ok && n % vw == 0 && (d->lda * eb) % 16 == 0 && (!d->B || (d->ldb * 4) % 16 == 0) &&
                         aligned16({d->A, d->B, d->u1, d->v1, d->u2, d->v2, d->y, d->x});
    if ((d->flags & CSPB_GEMVER_BULK) && !(d->flags & CSPB_GEMVER_PANEL) && bulk_ok) {
        GemverK g{};
        g.p1 = p1;
        g.p2 = p2;
        g.ctrl = reinterpret_cast<uint32_t*>(ws);
        g.units = L.units;
        g.z = d->z;
        g.beta = d->beta;
        g.x = d->x;
        void* args[] = {&g};
        if (bf16) return launch_coop_bulk(k_gemver_bulk<__nv_bfloat16, false, 5>, args,
                                          Ring<__nv_bfloat16, 5>::total, zero, ws, st);
        if (from_B) return launch_coop_bulk(k_gemver_bulk<float, true, 6>, args, Ring<float, 6>::total, zero, ws, st);
        return launch_coop_bulk(k_gemver_bulk<float, false, 6>, args, Ring<float, 6>::total, zero, ws, st);
    }
    if (!(d->flags & CSPB_GEMVER_PANEL)) {
        GemverK g{};
        g.p1 = p1;
        g.p2 = p2;
        g.ctrl = reinterpret_cast<uint32_t*>(ws);
        g.units = L.units;
        g.z = d->z;
        g.beta = d->beta;
        g.x = d->x;
        void* args[] = {&g, const_cast<int*>(&vec_ok)};
        if (bf16) return launch_coop(k_gemver<__nv_bfloat16, false>, args, L.units, zero, ws, st);
        if (from_B) return launch_coop(k_gemver<float, true>, args, L.units, zero, ws, st);
        return launch_coop(k_gemver<float, false>, args, L.units, zero, ws, st);
    }
    PanelK g{};
    g.p1 = p1;
    g.p2 = p2;
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    g.chunk_done = reinterpret_cast<uint32_t*>(ws + L.off_chunk);
    g.x_ready = g.chunk_done + L.chunks;
    g.z = d->z;
    g.beta = d->beta;
    g.x = d->x;
    // Pass 2 over panel c is queued `lag` panels after pass 1 over it. The blocks in flight hold about grid/S panels'
    // worth of pass-1 units, so a lag past that lets panel c finish before its pass 2 is taken (no waiting), while
    // the lag+1 panels of Â between the two reads stay well inside L2. Flags bits 8..15 override it (tuning).
    void* args[] = {&g, const_cast<int*>(&vec_ok)};
    const int64_t items = 2 * L.units;
    auto kern = bf16 ? k_gemver_panel<__nv_bfloat16, false>
                     : (from_B ? k_gemver_panel<float, true> : k_gemver_panel<float, false>);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPassThreads, 0) != cudaSuccess || per_sm < 1)
        return CSPB_ERR_LAUNCH;
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    const int64_t grid = int64_t(per_sm) * di.sms;
    const int64_t user_lag = (d->flags & CSPB_GEMVER_LAG_MASK) >> 8;
    int64_t lag = user_lag > 0 ? user_lag : (grid + L.strips - 1) / L.strips + 1;
    if (lag > L.chunks) lag = L.chunks;
    g.lag = lag;
    return launch_persistent(kern, args, items, zero, ws, st);
}

size_t cspb_bicgk_workspace_bytes(int64_t n) {
    if (n < 1) return 0;
    return pass_layout(n, kS, kCW32, 1, false).total;
}

int cspb_bicgk_fused(const cspb_bicgk_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    const int64_t n = d->n;
    if (n < 1 || d->ldb < n || n > (int64_t(1) << 31)) return CSPB_ERR_ARGUMENT;
    if (!d->B || !d->p || !d->r || !d->q || !d->s) return CSPB_ERR_ARGUMENT;
    if (d->b_dtype != CSPB_F32 && d->b_dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    if (d->flags != 0) return CSPB_ERR_UNSUPPORTED;
    const bool bf16 = d->b_dtype == CSPB_BF16;
    const PassLayout L = pass_layout(n, kS, bf16 ? kCW16 : kCW32, 1, false);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    char* ws = static_cast<char*>(d->workspace);
    BicgkK g{};
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    g.units = L.units;
    g.s = d->s;
    PassArgs& p = g.p;
    p.n = n;
    p.rows = n;
    p.src = d->B;
    p.lds = d->ldb;
    p.cyB = d->r;
    p.PB = reinterpret_cast<double*>(ws + L.off_PB);
    p.xv = d->p;
    p.Wp = reinterpret_cast<float*>(ws + L.off_Wp);
    p.strip_done = reinterpret_cast<uint32_t*>(ws + L.off_done);
    p.rout1 = d->q;
    p.rscale1 = 1.0f;
    p.strips = L.strips;
    p.chunks = L.chunks;
    const int vec_ok = vec_aligned(d->B, d->ldb, bf16 ? 2 : 4) ? 1 : 0;
    void* args[] = {&g, const_cast<int*>(&vec_ok)};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (bf16) return launch_coop(k_bicgk<__nv_bfloat16>, args, L.units, L.off_PA, ws, st);
    return launch_coop(k_bicgk<float>, args, L.units, L.off_PA, ws, st);
}

size_t cspb_chain_workspace_bytes(int64_t n) {
    if (n < 1) return 0;
    return pass_layout(n, kS, kCW32, 2, true).total;
}

int cspb_gemver_chain(const cspb_chain_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    const int64_t n = d->n;
    if (n < 1 || n > (int64_t(1) << 31)) return CSPB_ERR_ARGUMENT;
    const void* need[] = {d->A0, d->u1a, d->v1a, d->u2a, d->v2a, d->ya, d->u1b, d->v1b, d->u2b, d->v2b,
                          d->B1, d->x1, d->w1, d->q, d->s, d->B2, d->x2, d->w2};
    for (const void* p : need)
        if (!p) return CSPB_ERR_ARGUMENT;
    const PassLayout L = pass_layout(n, kS, kCW32, 2, true);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    char* ws = static_cast<char*>(d->workspace);
    ChainK g{};
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    g.units = L.units;
    g.za = d->za;
    g.beta = d->beta;
    g.x1 = d->x1;
    g.s = d->s;
    g.x2 = d->x2;
    uint32_t* done = reinterpret_cast<uint32_t*>(ws + L.off_done);
    double* PA = reinterpret_cast<double*>(ws + L.off_PA);
    double* PB = reinterpret_cast<double*>(ws + L.off_PB);
    float* Wp = reinterpret_cast<float*>(ws + L.off_Wp);
    PassArgs base{};
    base.n = n;
    base.rows = n;
    base.lds = n;
    base.ldd = n;
    base.strips = L.strips;
    base.chunks = L.chunks;
    // 1
    g.p1 = base;
    g.p1.src = d->A0;
    g.p1.dst = d->B1;
    g.p1.u1 = d->u1a; g.p1.v1 = d->v1a; g.p1.u2 = d->u2a; g.p1.v2 = d->v2a;
    g.p1.cyB = d->ya;
    g.p1.PB = PB;
    // 2
    g.p2 = base;
    g.p2.src = d->B1;
    g.p2.xv = d->x1;
    g.p2.Wp = Wp;
    g.p2.strip_done = done;
    g.p2.rout1 = d->w1;
    g.p2.rscale1 = d->alpha;
    g.p2.rout2 = d->q;
    g.p2.rscale2 = 1.0f;
    // 3
    g.p3 = base;
    g.p3.src = d->B1;
    g.p3.dst = d->B2;
    g.p3.u1 = d->u1b; g.p3.v1 = d->v1b; g.p3.u2 = d->u2b; g.p3.v2 = d->v2b;
    g.p3.cyA = d->w1;
    g.p3.PA = PA;
    g.p3.cyB = d->q;
    g.p3.PB = PB;
    // 4
    g.p4 = base;
    g.p4.src = d->B2;
    g.p4.xv = d->x2;
    g.p4.Wp = Wp;
    g.p4.strip_done = done + L.strips;
    g.p4.rout1 = d->w2;
    g.p4.rscale1 = d->alpha;
    const int vec_ok = (vec_aligned(d->A0, n, 4) && vec_aligned(d->B1, n, 4) && vec_aligned(d->B2, n, 4)) ? 1 : 0;
    void* args[] = {&g, const_cast<int*>(&vec_ok)};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the second launch reuses the first one's control block: its work counters were zeroed with the first
    int rc = launch_coop(k_chain_g1, args, L.units, L.off_PA, ws, st);
    if (rc != CSPB_OK) return rc;
    const size_t mbytes = size_t(n) * size_t(n) * sizeof(float);
    const char* b1 = reinterpret_cast<const char*>(d->B1);
    const char* b2 = reinterpret_cast<const char*>(d->B2);
    const bool disjoint = b1 + mbytes <= b2 || b2 + mbytes <= b1;
    return disjoint ? launch_coop(k_chain_g2<true>, args, L.units, 0, ws, st)
                    : launch_coop(k_chain_g2<false>, args, L.units, 0, ws, st);
}

// ---- row shards ------------------------------------------------------------------------------------------------

static PassLayout rows_layout(int64_t n, int64_t rows) {
    PassLayout L = pass_layout(n, kS, kCW32, 1, false);  // chunks and the column-length arrays follow n
    const int64_t strips = (rows + kS - 1) / kS;
    L.strips = strips;
    L.units = strips * L.chunks;
    return L;
}

size_t cspb_gemver_rows_workspace_bytes(int64_t n, int64_t rows) {
    if (n < 1 || rows < 1 || rows > n) return 0;
    return rows_layout(n, rows).total;
}

static int rows_args(const cspb_gemver_rows_desc* d, bool finish, RowsK& g, PassLayout& L, int& vec_ok, bool& bf16) {
    if (!d) return CSPB_ERR_ARGUMENT;
    const int64_t n = d->n, rows = d->rows;
    if (n < 1 || n > (int64_t(1) << 31) || rows < 1 || rows > n) return CSPB_ERR_ARGUMENT;
    if (d->a_dtype != CSPB_F32 && d->a_dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    if (d->flags != 0) return CSPB_ERR_UNSUPPORTED;
    if (!d->A || !d->u1 || !d->v1 || !d->u2 || !d->v2 || !d->y) return CSPB_ERR_ARGUMENT;
    if (finish && (!d->x || !d->w)) return CSPB_ERR_ARGUMENT;
    if (d->lda < n || (d->B && d->ldb < n)) return CSPB_ERR_ARGUMENT;
    L = rows_layout(n, rows);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    bf16 = d->a_dtype == CSPB_BF16;
    char* ws = static_cast<char*>(d->workspace);
    PassArgs p{};
    p.n = n;
    p.rows = rows;
    p.strips = L.strips;
    p.chunks = L.chunks;
    p.src = d->A;
    p.lds = d->lda;
    p.u1 = d->u1; p.v1 = d->v1; p.u2 = d->u2; p.v2 = d->v2;
    if (!finish) {
        p.dst = d->B;
        p.ldd = d->ldb;
        p.cyB = d->y;
        p.PB = reinterpret_cast<double*>(ws + L.off_PB);
    } else {
        if (!bf16 && d->B) {
            p.src = d->B;
            p.lds = d->ldb;
        }
        p.xv = d->x;
        p.Wp = reinterpret_cast<float*>(ws + L.off_Wp);
        p.strip_done = reinterpret_cast<uint32_t*>(ws + L.off_done);
        p.rout1 = d->w;
        p.rscale1 = d->alpha;
    }
    g = RowsK{};
    g.p = p;
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    g.units = L.units;
    g.z = d->z;
    g.beta = d->beta;
    g.x = d->x;
    const int eb = bf16 ? 2 : 4;
    vec_ok = vec_aligned(d->A, d->lda, eb) && vec_aligned(d->B, d->ldb, 4) ? 1 : 0;
    return CSPB_OK;
}

int cspb_gemver_rows_partial(const cspb_gemver_rows_desc* d, double* colsum, void* stream) {
    RowsK g;
    PassLayout L;
    int vec_ok = 0;
    bool bf16 = false;
    const int rc = rows_args(d, false, g, L, vec_ok, bf16);
    if (rc != CSPB_OK) return rc;
    if (!colsum) return CSPB_ERR_ARGUMENT;
    g.colsum = colsum;
    void* args[] = {&g, &vec_ok};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (bf16) return launch_coop(k_rows_partial<__nv_bfloat16>, args, L.units, L.off_PA, d->workspace, st);
    return launch_coop(k_rows_partial<float>, args, L.units, L.off_PA, d->workspace, st);
}

int cspb_gemver_rows_finish(const cspb_gemver_rows_desc* d, const double* colsum_total, void* stream) {
    RowsK g;
    PassLayout L;
    int vec_ok = 0;
    bool bf16 = false;
    const int rc = rows_args(d, true, g, L, vec_ok, bf16);
    if (rc != CSPB_OK) return rc;
    if (!colsum_total) return CSPB_ERR_ARGUMENT;
    g.total = colsum_total;
    void* args[] = {&g, &vec_ok};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t units = L.units > L.chunks ? L.units : L.chunks;  // the x phase wants blocks too
    if (bf16) return launch_coop(k_rows_finish<__nv_bfloat16, false>, args, units, L.off_PA, d->workspace, st);
    if (d->B) return launch_coop(k_rows_finish<float, true>, args, units, L.off_PA, d->workspace, st);
    return launch_coop(k_rows_finish<float, false>, args, units, L.off_PA, d->workspace, st);
}

}  // extern "C"
