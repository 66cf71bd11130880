// rowpass.cuh — the streaming matrix pass every GEMVER-family kernel of libcspb is built from.
//
// A pass walks an n×n row-major matrix in UNITS of S rows × CW columns (a strip × a column chunk). A 256-thread block
// owns one unit at a time: its 8 warps form a WX × WY grid, each warp covers 32 rows × (32 · VEC) columns, each lane
// VEC consecutive columns (one 16-byte load per row: 4 f32 or 8 bf16). Per loaded row a lane can
//   - add the rank-2 update (a + u1[i]·v1[j]) + u2[i]·v2[j]   (Rank2Update, examples/gemver-chain/components.hpp:85-97)
//   - store the updated row                                    (the B / Â output)
//   - accumulate column sums Σ_i a[i][j]·cyA[i] and Σ_i b[i][j]·cyB[i] in f64 (GemvTPartial + ColReduce,
//     components.hpp:142-219, and BicgkOnePass's Ps, components.hpp:306-320)
//   - form row dots Σ_j b[i][j]·xv[j]                           (Gemv, components.hpp:237-265; BicgkOnePass's Pq)
// Column sums leave the unit as one f64 partial per (strip, column); row dots as one f32 partial per (chunk, row),
// and the block that completes the last chunk of a strip combines them into the row results. Every sum runs in an
// order fixed by (n, S, CW) alone — never by the grid size, the scheduling or other work on the GPU — so a result is
// bit-identical however it was launched.
#pragma once

#include "common.cuh"

namespace cspb {

template <typename T> struct VecOf;
template <> struct VecOf<float> { static constexpr int N = 4; static constexpr int RB = 8; };
template <> struct VecOf<__nv_bfloat16> { static constexpr int N = 8; static constexpr int RB = 8; };

constexpr int kPassThreads = 256;
constexpr unsigned kFull = 0xffffffffu;

// Geometry of a pass (WX warps across columns).
template <typename T, int WX>
struct PassGeo {
    static constexpr int VEC = VecOf<T>::N;
    static constexpr int WY = 8 / WX;
    static constexpr int S = WY * 32;        // rows per strip
    static constexpr int CW = WX * 32 * VEC; // columns per chunk
};

struct PassArgs {
    int64_t n;         // columns (and the stride of PA / PB / Wp)
    int64_t rows;      // rows: n, except for a row shard of a larger GEMVER (sharded.cu)
    const void* src;   // the matrix read (T, or f32 when the pass reads B)
    int64_t lds;
    float* dst;        // STORE target (f32); NULL: no store
    int64_t ldd;
    const float *u1, *v1, *u2, *v2;  // rank-2 update
    const float* cyA;  // column sums of the loaded values, weighted per row
    double* PA;        // [strips][n]
    const float* cyB;  // column sums of the updated values
    double* PB;        // [strips][n]
    const float* xv;   // row dots with this column vector
    float* Wp;         // [chunks][n]
    uint32_t* strip_done;  // [strips]
    float* rout1;      // row results: rout1[i] = rscale1 · Σ_j b[i][j] xv[j]
    float rscale1;
    float* rout2;      // optional second copy with its own scale
    float rscale2;
    int64_t strips, chunks;
};

// 32 values per lane -> lane L holds the warp-wide sum of value L (31 shuffles, a fixed tree).
__device__ __forceinline__ float transpose_reduce32(float (&v)[32]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        const bool upper = (lane & off) != 0;
#pragma unroll
        for (int k = 0; k < off; ++k) {
            const float send = upper ? v[k] : v[k + off];
            const float keep = upper ? v[k + off] : v[k];
            v[k] = keep + __shfl_xor_sync(kFull, send, off);
        }
    }
    return v[0];
}

// One lane's VEC elements of a row as ONE raw 16-byte vector (4 f32 or 8 bf16), so that a batch of rows in flight
// costs 4 registers per row whatever the dtype; unpack() turns it into floats when the row is used. NC: the matrix is
// read-only for the whole kernel (an input), so the non-coherent path with evict-first is allowed; otherwise (a
// matrix written earlier in the same kernel) the load goes through L2 coherently. Lanes at the matrix edge (or rows
// that are not 16-byte aligned) load element by element into the same raw layout, zero-filled.
template <typename T, bool NC>
__device__ __forceinline__ uint4 load_raw(const T* row, int64_t c0, int ncols, bool vec_ok) {
    constexpr int VEC = VecOf<T>::N;
    if (vec_ok && ncols == VEC) {
        if constexpr (NC) return ld_stream_u4(row + c0);
        else {
            const float4 f = ld_cg_f4(reinterpret_cast<const float*>(row + c0));
            return make_uint4(__float_as_uint(f.x), __float_as_uint(f.y), __float_as_uint(f.z), __float_as_uint(f.w));
        }
    }
    uint32_t w[4] = {0u, 0u, 0u, 0u};
    if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int e = 0; e < 4; ++e)
            if (e < ncols) w[e] = __float_as_uint(NC ? __ldg(reinterpret_cast<const float*>(row) + c0 + e)
                                                     : __ldcg(reinterpret_cast<const float*>(row) + c0 + e));
    } else {
        const unsigned short* h = reinterpret_cast<const unsigned short*>(row) + c0;
#pragma unroll
        for (int e = 0; e < 8; ++e)
            if (e < ncols) w[e >> 1] |= uint32_t(h[e]) << (16 * (e & 1));
    }
    return make_uint4(w[0], w[1], w[2], w[3]);
}

template <typename T>
__device__ __forceinline__ void unpack(const uint4& v, float (&out)[VecOf<T>::N]) {
    if constexpr (sizeof(T) == 4) {
        out[0] = __uint_as_float(v.x); out[1] = __uint_as_float(v.y);
        out[2] = __uint_as_float(v.z); out[3] = __uint_as_float(v.w);
    } else {
        out[0] = bf16_lo(v.x); out[1] = bf16_hi(v.x); out[2] = bf16_lo(v.y); out[3] = bf16_hi(v.y);
        out[4] = bf16_lo(v.z); out[5] = bf16_hi(v.z); out[6] = bf16_lo(v.w); out[7] = bf16_hi(v.w);
    }
}

template <int VEC>
__device__ __forceinline__ void store_vec(float* row, int64_t c0, int ncols, bool vec_ok, const float (&b)[VEC]) {
    if (vec_ok && ncols == VEC) {
#pragma unroll
        for (int q = 0; q < VEC / 4; ++q) st_f4(row + c0 + 4 * q, make_float4(b[4 * q], b[4 * q + 1], b[4 * q + 2], b[4 * q + 3]));
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e)
            if (e < ncols) row[c0 + e] = b[e];
    }
}

// 16-bit storage carries twice the elements per byte: its column sums take 8 products in f32 before each f64
// addition, so that the f32 -> f64 conversions do not bound the pass (f32 storage converts every product).
template <typename LT> inline constexpr bool kF32Part = sizeof(LT) == 2;

// 16-bit storage also keeps its unit loop rolled (8 rows of 8 elements per lane and batch make a fully unrolled unit
// too large for the instruction cache); its row dots then wait in shared memory, one float per (warp, row, lane),
// in the same region the epilogue uses afterwards.
template <typename LT> inline constexpr bool kRolled = sizeof(LT) == 2;
constexpr size_t kRolledDotBytes = size_t(kPassThreads) * 32 * sizeof(float);

// Shared memory a pass needs (bytes).
template <typename T, int WX>
__host__ __device__ constexpr size_t pass_smem_bytes() {
    using G = PassGeo<T, WX>;
    const size_t cs = size_t(G::WY) * G::CW * sizeof(double);
    const size_t rd = size_t(WX) * G::S * sizeof(float);
    const size_t m = cs > rd ? cs : rd;
    return kRolled<T> && kRolledDotBytes > m ? kRolledDotBytes : m;
}

// Synchronisation of the threads that run a unit's epilogue: the whole block (pass_unit) or, in a kernel with a
// producer warp, the 256 consumer threads only (named barrier 1).
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct ConsumerSync {
    __device__ __forceinline__ void operator()() const { asm volatile("bar.sync 1, 256;" ::: "memory"); }
};

// The end of a unit, run by threads 0..255: column sums (the WY warps of a column combined in a fixed order, one f64
// partial per (strip, column)) and row dots (warp tree, then the WX warps of a row in order; the last chunk of a strip
// combines the chunks in order and writes the row results). Every order here depends on (n, S, CW) only.
// DEFER: the row dots stop at the per-chunk partials (Wp); rowsum_finish combines them after a grid barrier, in the
// same order, so the unit ends without a fence, an atomic and the last block's sums.
template <typename LT, int WX, bool CSA, bool CSB, bool RDOT, typename Sync, bool DEFER = false>
__device__ __forceinline__ void unit_epilogue(const PassArgs& a, int64_t strip, int64_t chunk,
                                              const double (&accA)[VecOf<LT>::N], const double (&accB)[VecOf<LT>::N],
                                              float (&racc)[32], unsigned char* smem, Sync sync) {
    using G = PassGeo<LT, WX>;
    constexpr int VEC = G::VEC, WY = G::WY, S = G::S, CW = G::CW;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wx = warp % WX, wy = warp / WX;
    const int64_t n = a.n;
    __shared__ int s_last;
    if (CSA || CSB) {
        double* red = reinterpret_cast<double*>(smem);
#pragma unroll
        for (int which = 0; which < 2; ++which) {
            if ((which == 0 && !CSA) || (which == 1 && !CSB)) continue;
            sync();
#pragma unroll
            for (int e = 0; e < VEC; ++e) red[wy * CW + (wx * 32 + lane) * VEC + e] = which == 0 ? accA[e] : accB[e];
            sync();
            double* P = which == 0 ? a.PA : a.PB;
            for (int t = threadIdx.x; t < CW; t += kPassThreads) {
                const int64_t col = chunk * CW + t;
                if (col < n) {
                    double s = red[t];
#pragma unroll
                    for (int y = 1; y < WY; ++y) s += red[y * CW + t];
                    P[strip * n + col] = s;
                }
            }
        }
    }
    if (RDOT) {
        const float v = transpose_reduce32(racc);
        float* red2 = reinterpret_cast<float*>(smem);
        sync();
        red2[wx * S + wy * 32 + lane] = v;
        sync();
        for (int t = threadIdx.x; t < S; t += kPassThreads) {
            const int64_t row = strip * S + t;
            if (row < a.rows) {
                float s = red2[t];
#pragma unroll
                for (int x = 1; x < WX; ++x) s += red2[x * S + t];
                a.Wp[chunk * n + row] = s;
            }
        }
        if (DEFER) return;
        // the last block of the strip: one thread fences after the barrier, for the whole block (the pattern of a
        // cooperative grid sync: the barrier orders the other threads' partials before that fence)
        sync();
        if (threadIdx.x == 0) {
            __threadfence();
            s_last = atomicAdd(a.strip_done + strip, 1u) == uint32_t(a.chunks - 1);
            if (s_last) __threadfence();
        }
        sync();
        if (s_last) {
            for (int t = threadIdx.x; t < S; t += kPassThreads) {
                const int64_t row = strip * S + t;
                if (row < a.rows) {
                    // chunks in order; 16 loads in flight at a time (the partials sit in L2)
                    float s = 0.f;
                    int64_t c = 0;
                    for (; c + 16 <= a.chunks; c += 16) {
                        float v[16];
#pragma unroll
                        for (int q = 0; q < 16; ++q) v[q] = __ldcg(a.Wp + (c + q) * n + row);
#pragma unroll
                        for (int q = 0; q < 16; ++q) s += v[q];
                    }
                    for (; c < a.chunks; ++c) s += __ldcg(a.Wp + c * n + row);
                    a.rout1[row] = a.rscale1 * s;
                    if (a.rout2) a.rout2[row] = a.rscale2 * s;
                }
            }
        }
    }
}

// One unit of a pass. LT: the loaded element type; NC: see load_vec. Flags: RANK2 add the update; CSA / CSB column sums of the loaded /
// updated values; RDOT row dots of the updated values. Stores happen when a.dst != NULL. RBX: rows each lane keeps in
// flight (0: VecOf's default; only the batching changes, not the arithmetic). DEFER: see unit_epilogue.
template <typename LT, int WX, bool NC, bool RANK2, bool CSA, bool CSB, bool RDOT, int RBX = 0, bool DEFER = false>
__device__ __forceinline__ void pass_unit(const PassArgs& a, int64_t unit, bool vec_ok, unsigned char* smem) {
    using G = PassGeo<LT, WX>;
    constexpr int VEC = G::VEC, WY = G::WY, S = G::S, CW = G::CW, RB = RBX ? RBX : VecOf<LT>::RB;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wx = warp % WX, wy = warp / WX;
    const int64_t n = a.n;
    const int64_t strip = unit / a.chunks, chunk = unit % a.chunks;
    const int64_t r0 = strip * S + wy * 32;
    const int64_t c0 = chunk * CW + int64_t(wx * 32 + lane) * VEC;
    const int64_t rem_r = a.rows - r0, rem_c = n - c0;
    const int nrows = rem_r <= 0 ? 0 : (rem_r >= 32 ? 32 : int(rem_r));
    const int ncols = rem_c <= 0 ? 0 : (rem_c >= VEC ? VEC : int(rem_c));

    float u1r = 0.f, u2r = 0.f, cyar = 0.f, cybr = 0.f;
    if (lane < nrows) {
        const int64_t row = r0 + lane;
        if (RANK2) { u1r = __ldcg(a.u1 + row); u2r = __ldcg(a.u2 + row); }
        if (CSA) cyar = __ldcg(a.cyA + row);
        if (CSB) cybr = __ldcg(a.cyB + row);
    }
    float v1c[VEC], v2c[VEC], xc[VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) {
        const bool ok = e < ncols;
        v1c[e] = (RANK2 && ok) ? __ldcg(a.v1 + c0 + e) : 0.f;
        v2c[e] = (RANK2 && ok) ? __ldcg(a.v2 + c0 + e) : 0.f;
        xc[e] = (RDOT && ok) ? __ldcg(a.xv + c0 + e) : 0.f;
    }
    double accA[VEC], accB[VEC];
#pragma unroll
    for (int e = 0; e < VEC; ++e) { accA[e] = 0.0; accB[e] = 0.0; }
    float pA[VEC], pB[VEC];  // f32 partials of 8 rows (16-bit storage only)
#pragma unroll
    for (int e = 0; e < VEC; ++e) { pA[e] = 0.f; pB[e] = 0.f; }
    float racc[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) racc[k] = 0.f;

    // the arguments the row loop uses, in registers: `a` may live in shared memory (a persistent caller's cached
    // instance), which the loop's own shared-memory stores would otherwise make the compiler read again
    const LT* src = static_cast<const LT*>(a.src);
    const int64_t lds = a.lds, ldd = a.ldd;
    float* const dst = a.dst;
    const bool store = dst != nullptr;
    float* rdot = reinterpret_cast<float*>(smem) + size_t(warp) * 32 * 32;  // rolled loop: [row][lane] of the warp

    auto batch = [&](int kb) {
        if (kb < nrows) {  // warp-uniform
            uint4 raw[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k)
                raw[k] = (kb + k < nrows && ncols > 0) ? load_raw<LT, NC>(src + (r0 + kb + k) * lds, c0, ncols, vec_ok)
                                                       : make_uint4(0u, 0u, 0u, 0u);
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                const int kk = kb + k;
                const float u1k = __shfl_sync(kFull, u1r, kk);
                const float u2k = __shfl_sync(kFull, u2r, kk);
                const float cyak = __shfl_sync(kFull, cyar, kk);
                const float cybk = __shfl_sync(kFull, cybr, kk);
                if (kk < nrows) {
                    float val[VEC];
                    unpack<LT>(raw[k], val);
                    float b[VEC];
#pragma unroll
                    for (int e = 0; e < VEC; ++e)
                        b[e] = RANK2 ? __fadd_rn(__fadd_rn(val[e], __fmul_rn(u1k, v1c[e])), __fmul_rn(u2k, v2c[e]))
                                     : val[e];
                    if (store && ncols > 0) store_vec<VEC>(dst + (r0 + kk) * ldd, c0, ncols, vec_ok, b);
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
                        if constexpr (kRolled<LT>) rdot[kk * 32 + lane] = d;
                        else racc[kk] = d;
                    }
                }
            }
        }
    };
    if constexpr (kRolled<LT>) {
#pragma unroll 1
        for (int kb = 0; kb < 32; kb += RB) batch(kb);
        if (RDOT) {
#pragma unroll
            for (int k = 0; k < 32; ++k) racc[k] = k < nrows ? rdot[k * 32 + lane] : 0.f;  // this lane's own values
        }
    } else {
#pragma unroll
        for (int kb = 0; kb < 32; kb += RB) batch(kb);
    }

    unit_epilogue<LT, WX, CSA, CSB, RDOT, BlockSync, DEFER>(a, strip, chunk, accA, accB, racc, smem, BlockSync{});
}

// rout1[row] = rscale1 · Σ_c Wp[c][row] over the chunks in index order (f32: the order of unit_epilogue's last
// block, so a deferred pass gives the same bits), and rout2 likewise; by every thread of the grid, no barrier inside.
__device__ __forceinline__ void rowsum_finish(const PassArgs& a) {
    const int64_t gthreads = int64_t(gridDim.x) * blockDim.x;
    for (int64_t row = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; row < a.rows; row += gthreads) {
        float s = 0.f;
        int64_t c = 0;
        for (; c + 16 <= a.chunks; c += 16) {
            float v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = __ldcg(a.Wp + (c + q) * a.n + row);
#pragma unroll
            for (int q = 0; q < 16; ++q) s += v[q];
        }
        for (; c < a.chunks; ++c) s += __ldcg(a.Wp + c * a.n + row);
        a.rout1[row] = a.rscale1 * s;
        if (a.rout2) a.rout2[row] = a.rscale2 * s;
    }
}

// Σ P[st][j] over st = q, q+4, q+8, ... < strips, in that order, with 8 loads in flight.
__device__ __forceinline__ double strided_strip_sum(const double* P, int64_t strips, int64_t n, int64_t j, int q) {
    double s = 0.0;
    int64_t st = q;
    for (; st + 28 < strips; st += 32) {
        double v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldcg(P + (st + 4 * k) * n + j);
#pragma unroll
        for (int k = 0; k < 8; ++k) s += v[k];
    }
    for (; st < strips; st += 4) s += __ldcg(P + st * n + j);
    return s;
}

// out[j] = (z ? z[j] : 0) + scale · Σ_s P[s][j] over all strips in index order (f64), rounded once to f32.
// Four lanes share a column: lane q sums strips q, q+4, ...; the four partials combine as ((p0+p1)+(p2+p3)).
// Called by every thread of the grid; no barrier inside.
__device__ __forceinline__ void colsum_finish(const double* P, int64_t strips, int64_t n, const float* z, float scale,
                                              float* out) {
    const int lane = threadIdx.x & 31;
    const int64_t gthreads = int64_t(gridDim.x) * blockDim.x;
    const int64_t gtid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t base = gtid - lane; base < 4 * n; base += gthreads) {
        const int64_t item = base + lane;
        const bool valid = item < 4 * n;
        const int64_t j = item >> 2;
        const int q = int(item & 3);
        double s = valid ? strided_strip_sum(P, strips, n, j, q) : 0.0;
        s += __shfl_xor_sync(kFull, s, 1);
        s += __shfl_xor_sync(kFull, s, 2);
        if (valid && q == 0) {
            const double zz = z ? double(__ldcg(z + j)) : 0.0;
            out[j] = float(zz + double(scale) * s);
        }
    }
}

// The same sums for the columns [c0, c1) only, by the threads of ONE block (the identical order, so a result formed
// here is bit-identical to one formed by colsum_finish).
__device__ __forceinline__ void colsum_finish_cols(const double* P, int64_t strips, int64_t n, int64_t c0, int64_t c1,
                                                   const float* z, float scale, float* out) {
    const int lane = threadIdx.x & 31;
    const int64_t items = 4 * (c1 - c0);
    for (int64_t base = int64_t(threadIdx.x) - lane; base < items; base += blockDim.x) {
        const int64_t item = base + lane;
        const bool valid = item < items;
        const int64_t j = c0 + (item >> 2);
        const int q = int(item & 3);
        double s = valid ? strided_strip_sum(P, strips, n, j, q) : 0.0;
        s += __shfl_xor_sync(kFull, s, 1);
        s += __shfl_xor_sync(kFull, s, 2);
        if (valid && q == 0) {
            const double zz = z ? double(__ldcg(z + j)) : 0.0;
            out[j] = float(zz + double(scale) * s);
        }
    }
}

// a·b and c·b over [0, n) in f64, formed by ONE block in a fixed order (thread-strided sums, then a fixed tree), so
// every block of a grid that calls it gets the same two values. For the low-rank GEMVER's finishes.
__device__ __forceinline__ void block_dot2(const float* a, const float* c, const float* b, int64_t n, double& ab,
                                           double& cb) {
    __shared__ double s_red[2][kPassThreads / 32];
    double s0 = 0.0, s1 = 0.0;
    for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
        const double bj = double(__ldcg(b + j));
        s0 = __fma_rn(double(__ldcg(a + j)), bj, s0);
        s1 = __fma_rn(double(__ldcg(c + j)), bj, s1);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        s0 += __shfl_xor_sync(kFull, s0, off);
        s1 += __shfl_xor_sync(kFull, s1, off);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) {
        s_red[0][warp] = s0;
        s_red[1][warp] = s1;
    }
    __syncthreads();
    double t0 = 0.0, t1 = 0.0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
        t0 += s_red[0][w];
        t1 += s_red[1][w];
    }
    ab = t0;
    cb = t1;
}

// x[j] = float(z[j] + scale·(Σ_strips P[st][j] + v1[j]·s1 + v2[j]·s2)): colsum_finish with the low-rank terms of
// Âᵀy = Aᵀy + v1(u1·y) + v2(u2·y) (s1 = u1·y, s2 = u2·y).
__device__ __forceinline__ void colsum_finish_lr(const double* P, int64_t strips, int64_t n, const float* z, float scale,
                                                 const float* v1, const float* v2, double s1, double s2, float* out) {
    const int lane = threadIdx.x & 31;
    const int64_t gthreads = int64_t(gridDim.x) * blockDim.x;
    const int64_t gtid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t base = gtid - lane; base < 4 * n; base += gthreads) {
        const int64_t item = base + lane;
        const bool valid = item < 4 * n;
        const int64_t j = item >> 2;
        const int q = int(item & 3);
        double s = valid ? strided_strip_sum(P, strips, n, j, q) : 0.0;
        s += __shfl_xor_sync(kFull, s, 1);
        s += __shfl_xor_sync(kFull, s, 2);
        if (valid && q == 0) {
            s = __fma_rn(double(__ldcg(v1 + j)), s1, s);
            s = __fma_rn(double(__ldcg(v2 + j)), s2, s);
            const double zz = z ? double(__ldcg(z + j)) : 0.0;
            out[j] = float(zz + double(scale) * s);
        }
    }
}

// w[i] = float(scale·(Σ_c Wp[c][i] + u1[i]·t1 + u2[i]·t2)): rowsum_finish with the low-rank terms of Â·x = A·x +
// u1(v1·x) + u2(v2·x) (t1 = v1·x, t2 = v2·x); the chunk sums in index order, in f32 as rowsum_finish, then f64.
__device__ __forceinline__ void rowsum_finish_lr(const PassArgs& a, const float* u1, const float* u2, double t1, double t2) {
    const int64_t gthreads = int64_t(gridDim.x) * blockDim.x;
    for (int64_t row = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; row < a.n; row += gthreads) {
        float s = 0.f;
        int64_t c = 0;
        for (; c + 16 <= a.chunks; c += 16) {
            float v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = __ldcg(a.Wp + (c + q) * a.n + row);
#pragma unroll
            for (int q = 0; q < 16; ++q) s += v[q];
        }
        for (; c < a.chunks; ++c) s += __ldcg(a.Wp + c * a.n + row);
        double d = double(s);
        d = __fma_rn(double(__ldcg(u1 + row)), t1, d);
        d = __fma_rn(double(__ldcg(u2 + row)), t2, d);
        a.rout1[row] = float(double(a.rscale1) * d);
    }
}

// out[j] = Σ_strips P[st][j] in f64 over every column, in colsum_finish's order (four strided sums, then pairs), not
// rounded: a row shard's share of the column sums, added across shards by the caller (sharded GEMVER).
__device__ __forceinline__ void colsum_f64(const double* P, int64_t strips, int64_t n, double* out) {
    const int lane = threadIdx.x & 31;
    const int64_t gthreads = int64_t(gridDim.x) * blockDim.x;
    const int64_t gtid = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    for (int64_t base = gtid - lane; base < 4 * n; base += gthreads) {
        const int64_t item = base + lane;
        const bool valid = item < 4 * n;
        const int64_t j = item >> 2;
        const int q = int(item & 3);
        double s = valid ? strided_strip_sum(P, strips, n, j, q) : 0.0;
        s += __shfl_xor_sync(kFull, s, 1);
        s += __shfl_xor_sync(kFull, s, 2);
        if (valid && q == 0) out[j] = s;
    }
}

}  // namespace cspb
