// ns_comp.cu — the reference's compressible Navier-Stokes residual and its diagnostics in ONE kernel.
//
// Reproduces examples/ns-residual: the physics of physics.hpp (to_prim :86-94, grad_cell :97-104, HLLC :109-152,
// visc_flux :157-192, cell_diag :196-202, MinMod / VanLeer :62-80), the tile stages of tile.hpp:39-229, and the
// diagnostics of components.hpp:393-628 (atomic min dt / max wave speed / Σ R², their deterministic fixed-order
// counterparts, and the error stage atomic − deterministic).
//
// The reference's fused group (systems.hpp:88-140) and its hand-written kernel (handwritten.hpp:51-191) write the four
// face-flux arrays to global memory and wait on neighbour tiles before the divergence (≈1 GiB round trip at 4096²).
// Here a block owns a 32×15 tile and keeps everything on chip: it loads the tile with a 2-cell halo (boundary rule
// applied on the fly), forms primitives in shared memory, evaluates every face of its cells once — two faces per
// thread, each value a pair whose lanes belong to the two faces, on Blackwell's packed f32x2 arithmetic — and writes
// R. The faces on the tile's east and north edges are evaluated by both neighbouring tiles with the same code, so R
// does not depend on the tiling. HBM traffic is one read of U and one write of R (32 B/cell); the halo re-reads are L2
// hits. The kernel is bound by instruction issue, not by HBM (about 0.51 ms at 4096² against 0.08 ms of traffic).
//
// Two arithmetic forms (Ar<X>): the fast one (fused multiply-adds, approximate reciprocal / square root / division in
// the face fluxes) and the reference's rounding (every operation rounded as physics.hpp writes it, IEEE division and
// square root), whose R and per-cell dt / wave speed are bit-identical to a sequential f32 evaluation of physics.hpp.
//
// Diagnostics: per tile, min dt, max wave speed and Σ R² (f64) in a fixed order; atomics for the atomic path (integer
// max on the bit patterns of positive floats for min / max, float add of the tile's sum rounded to f32); per-tile
// partials, and the last block to finish reduces them in tile order (min / max exactly, sums in f64) and writes the
// error stage. Deterministic results are bit-identical on every run.
#include "common.cuh"

namespace cspb {
namespace nsc {

constexpr int TX = 32, TY = 15;              // tile of cells: 16 rows of y-faces, two per thread (rows f, f + 8)
constexpr int LX = TX + 4, LY = TY + 4;      // with the 2-cell halo
constexpr int LC = LX * LY;                  // 720
constexpr int NXF = (TX + 1) * TY;           // x-faces of the tile's rows
constexpr int NYF = TX * (TY + 1);           // y-faces of the tile's columns
constexpr int kThreads = 256;

constexpr float kG = 1.4f, kMu = 0.01f, kPr = 0.72f, kCfl = 0.5f;
constexpr float kGm1 = kG - 1.0f;                   // γ - 1 in f32, as the reference's T(kGamma) - T(1)
constexpr float kInvGm1 = 1.0f / kGm1;              // its reciprocal, rounded once (fast arithmetic only)
constexpr float kKt = kMu * kG / (kGm1 * kPr);      // the heat conductivity μγ / ((γ - 1) Pr), as visc_flux forms it
constexpr float kTwo3 = 2.0f / 3.0f;
constexpr float kNuMax = (4.0f / 3.0f) > (kG / kPr) ? (4.0f / 3.0f) : (kG / kPr);  // tmax(4/3, γ / Pr)

// The tile's state in shared memory: primitives and temperature of the tile with its 2-cell halo, and both fluxes of
// every face. A face forms the gradients and limited slopes of its two cells from W and T itself.
struct Smem {
    float W[4][LC];    // primitives ρ u v p
    float T[LC];       // p / ρ
    float FX[8][NXF];  // HLLC 0..3, viscous 4..7
    float FY[8][NYF];
};
// the tile's end reuses T for 2 floats a thread and FX for 4 doubles a thread
static_assert(LC >= 2 * kThreads && 8 * NXF * sizeof(float) >= 4 * kThreads * sizeof(double) &&
                  (sizeof(float) * 5 * LC) % sizeof(double) == 0,
              "the tile's reduction fits T and FX, FX 8-byte aligned");

// ---- arithmetic on pairs of faces (or cells) ------------------------------------------------------------------------
// A thread evaluates two faces at once: every value is a float2 whose lanes belong to the two faces, and the adds,
// multiplies and fused multiply-adds are Blackwell's packed f32x2 instructions (FADD2 / FMUL2 / FFMA2), each lane
// rounded exactly as the scalar instruction would round it. Divisions, square roots, comparisons and selects act per
// lane. Ar<X> is the arithmetic policy:
//   X = false  the fast form: fused multiply-adds where they fit, approximate reciprocal / division / reciprocal square
//              root in the face fluxes (about 2 ulp);
//   X = true   the reference's rounding: the formulas of physics.hpp in their written order, every multiply and add
//              rounded separately (no fused multiply-add), IEEE division and square root. The residual is then
//              bit-identical to a sequential f32 evaluation of physics.hpp (the oracle's ns_comp_f32). This form
//              works lane by lane with __fadd_rn / __fsub_rn / __fmul_rn, which the compiler never merges into a
//              fused multiply-add; a subtraction written as a packed a + b·(-1) was merged with the multiply that
//              produced b in some faces, which changed the last bit.
using V = float2;
__device__ __forceinline__ V v2(float a, float b) { return make_float2(a, b); }
// the hardware's approximate reciprocal and square root (one MUFU instruction each; sqrt(0) = 0)
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
    float r;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ V sp(float a) { return make_float2(a, a); }

template <bool X>
struct Ar {
    static __device__ __forceinline__ V add(V a, V b) {
        if constexpr (X) return v2(__fadd_rn(a.x, b.x), __fadd_rn(a.y, b.y));
        else return __fadd2_rn(a, b);
    }
    // fast form: a - b as a + b·(-1) (one rounding; the compiler may fuse a multiply that produced b into it)
    static __device__ __forceinline__ V sub(V a, V b) {
        if constexpr (X) return v2(__fsub_rn(a.x, b.x), __fsub_rn(a.y, b.y));
        else return __ffma2_rn(b, sp(-1.0f), a);
    }
    static __device__ __forceinline__ V mul(V a, V b) {
        if constexpr (X) return v2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y));
        else return __fmul2_rn(a, b);
    }
    static __device__ __forceinline__ V fma(V a, V b, V c) {  // a·b + c
        if constexpr (X) return add(mul(a, b), c);
        else return __ffma2_rn(a, b, c);
    }
    // division: IEEE per lane, or (fast) the approximate reciprocal per lane times a, packed
    static __device__ __forceinline__ V div(V a, V b) {
        if constexpr (X) return v2(__fdiv_rn(a.x, b.x), __fdiv_rn(a.y, b.y));
        else return mul(a, rcp(b));
    }
    static __device__ __forceinline__ V rcp(V b) { return v2(rcp_approx(b.x), rcp_approx(b.y)); }
    // tmin / tmax of physics.hpp (a < b ? a : b); the fast form takes the min / max instructions
    static __device__ __forceinline__ float mn1(float a, float b) {
        if constexpr (X) return a < b ? a : b;
        else return fminf(a, b);
    }
    static __device__ __forceinline__ float mx1(float a, float b) {
        if constexpr (X) return a > b ? a : b;
        else return fmaxf(a, b);
    }
    static __device__ __forceinline__ V mn(V a, V b) { return v2(mn1(a.x, b.x), mn1(a.y, b.y)); }
    static __device__ __forceinline__ V mx(V a, V b) { return v2(mx1(a.x, b.x), mx1(a.y, b.y)); }
};

// The limited slope from the backward difference a and the forward difference b (MinMod / VanLeer, physics.hpp:62-80):
// zero at an extremum. MinMod returns whichever of a, b is nearer zero: the fast form as min(|a|, |b|) with a's sign.
template <int LIM, bool X>
__device__ __forceinline__ float minmod1(float a, float b, float ab) {
    if constexpr (X) {
        if (ab <= 0.0f) return 0.0f;
        return a > 0.0f ? (a < b ? a : b) : (a > b ? a : b);
    } else {
        return ab <= 0.0f ? 0.0f : copysignf(fminf(fabsf(a), fabsf(b)), a);
    }
}
template <int LIM, bool X>
__device__ __forceinline__ V slope2(V a, V b) {
    using A = Ar<X>;
    const V ab = A::mul(a, b);
    if constexpr (LIM == 0) {
        return v2(minmod1<LIM, X>(a.x, b.x, ab.x), minmod1<LIM, X>(a.y, b.y, ab.y));
    } else {
        const V q = A::div(A::mul(sp(2.0f), ab), A::add(a, b));
        return v2(ab.x <= 0.0f ? 0.0f : q.x, ab.y <= 0.0f ? 0.0f : q.y);
    }
}

__device__ __forceinline__ V sel(bool cx, bool cy, V a, V b) { return v2(cx ? a.x : b.x, cy ? a.y : b.y); }

// HLLC with Davis speeds through faces of normal D (0: x, 1: y); L / R the reconstructed primitives (ρ, u, v, p) of
// the two sides (physics.hpp:109-152). Per lane the region is chosen as the reference chooses it (sl >= 0: left state;
// sr <= 0: right state; else the star state of the side sm points to); the side state's flux is the first term of the
// star flux, so both regions share it and the star increment s·(…) is added where the face is in the star region.
template <int D, bool X>
__device__ __forceinline__ void hllc2(const V (&L)[4], const V (&R)[4], V (&F)[4]) {
    using A = Ar<X>;
    const V rl = L[0], rr = R[0], pl = L[3], pr = R[3];
    const V unl = L[1 + D], utl = L[2 - D];
    const V unr = R[1 + D], utr = R[2 - D];
    const V half = sp(0.5f);
    V cl, cr, El, Er, irl, irr;
    if constexpr (X) {
        const V gl = A::div(A::mul(sp(kG), pl), rl), gr = A::div(A::mul(sp(kG), pr), rr);
        cl = v2(__fsqrt_rn(gl.x), __fsqrt_rn(gl.y));
        cr = v2(__fsqrt_rn(gr.x), __fsqrt_rn(gr.y));
        El = A::add(A::div(pl, sp(kGm1)), A::mul(A::mul(half, rl), A::add(A::mul(unl, unl), A::mul(utl, utl))));
        Er = A::add(A::div(pr, sp(kGm1)), A::mul(A::mul(half, rr), A::add(A::mul(unr, unr), A::mul(utr, utr))));
        irl = irr = sp(0.0f);
    } else {
        irl = A::rcp(rl);
        irr = A::rcp(rr);
        const V gl = A::mul(A::mul(sp(kG), pl), irl), gr = A::mul(A::mul(sp(kG), pr), irr);
        cl = v2(sqrt_approx(gl.x), sqrt_approx(gl.y));
        cr = v2(sqrt_approx(gr.x), sqrt_approx(gr.y));
        El = A::fma(A::mul(half, rl), A::fma(unl, unl, A::mul(utl, utl)), A::mul(pl, sp(kInvGm1)));
        Er = A::fma(A::mul(half, rr), A::fma(unr, unr, A::mul(utr, utr)), A::mul(pr, sp(kInvGm1)));
    }
    const V sl = A::mn(A::sub(unl, cl), A::sub(unr, cr));
    const V sr = A::mx(A::add(unl, cl), A::add(unr, cr));
    const V al = A::sub(sl, unl), ar = A::sub(sr, unr);
    const V num = A::sub(A::fma(A::mul(rl, unl), al, A::sub(pr, pl)), A::mul(A::mul(rr, unr), ar));
    const V sm = A::div(num, A::sub(A::mul(rl, al), A::mul(rr, ar)));

    const bool supx = sl.x >= 0.0f, supy = sl.y >= 0.0f;        // supersonic to the right: the left state
    const bool subx = sr.x <= 0.0f, suby = sr.y <= 0.0f;        // supersonic to the left: the right state
    const bool lx = supx || (!subx && sm.x >= 0.0f), ly = supy || (!suby && sm.y >= 0.0f);
    const bool starx = !supx && !subx, stary = !supy && !suby;
    const V r = sel(lx, ly, rl, rr), un = sel(lx, ly, unl, unr), ut = sel(lx, ly, utl, utr);
    const V p = sel(lx, ly, pl, pr), E = sel(lx, ly, El, Er), s = sel(lx, ly, sl, sr);
    const V ru = A::mul(r, un);
    const V f0 = ru, f1 = A::fma(ru, un, p), f2 = A::mul(ru, ut), f3 = A::mul(A::add(E, p), un);
    const V a = A::sub(s, un);
    const V k = A::div(A::mul(r, a), A::sub(s, sm));
    V Es;
    if constexpr (X) {
        Es = A::mul(k, A::add(A::div(E, r), A::mul(A::sub(sm, un), A::add(sm, A::div(p, A::mul(r, a))))));
    } else {
        const V ir = sel(lx, ly, irl, irr);
        Es = A::mul(k, A::fma(A::sub(sm, un), A::add(sm, A::div(A::mul(p, ir), a)), A::mul(E, ir)));
    }
    const V g0 = A::fma(s, A::sub(k, r), f0);
    const V g1 = A::fma(s, A::sub(A::mul(k, sm), ru), f1);
    const V g2 = A::fma(s, A::sub(A::mul(k, ut), A::mul(r, ut)), f2);
    const V g3 = A::fma(s, A::sub(Es, E), f3);
    F[0] = sel(starx, stary, g0, f0);
    F[1 + D] = sel(starx, stary, g1, f1);
    F[2 - D] = sel(starx, stary, g2, f2);
    F[3] = sel(starx, stary, g3, f3);
}

// The viscous flux through faces of normal D (physics.hpp:157-192): the normal derivatives are the differences of the
// two cells; the tangential ones (dut, dvt, dTt) the means of the two cells' central differences.
template <int D, bool X>
__device__ __forceinline__ void visc2(const V (&L)[4], const V (&R)[4], V TL, V TR, V dut, V dvt, V dTt,
                                      V (&F)[4]) {
    using A = Ar<X>;
    const V half = sp(0.5f);
    const V uf = A::mul(half, A::add(L[1], R[1])), vf = A::mul(half, A::add(L[2], R[2]));
    V ux, uy, vx, vy, Tx, Ty;
    if (D == 0) {
        ux = A::sub(R[1], L[1]); vx = A::sub(R[2], L[2]); Tx = A::sub(TR, TL);
        uy = dut; vy = dvt; Ty = dTt;
    } else {
        uy = A::sub(R[1], L[1]); vy = A::sub(R[2], L[2]); Ty = A::sub(TR, TL);
        ux = dut; vx = dvt; Tx = dTt;
    }
    const V mu = sp(kMu), two = sp(2.0f);
    const V dv = A::add(ux, vy);
    const V t3 = A::mul(sp(kTwo3), dv);
    const V txx = A::mul(mu, A::sub(A::mul(two, ux), t3));
    const V tyy = A::mul(mu, A::sub(A::mul(two, vy), t3));
    const V txy = A::mul(mu, A::add(uy, vx));
    F[0] = sp(0.0f);
    if (D == 0) {
        F[1] = txx; F[2] = txy; F[3] = A::fma(sp(kKt), Tx, A::fma(vf, txy, A::mul(uf, txx)));
    } else {
        F[1] = txy; F[2] = tyy; F[3] = A::fma(sp(kKt), Ty, A::fma(vf, tyy, A::mul(uf, txy)));
    }
}

// Two faces of normal D, the first between smem cells ca and ca + st, the second between cb and cb + st (st the
// neighbour along the normal): the limited slopes of the four cells along the normal, the reconstructed states, the
// HLLC fluxes, the tangential gradients and the viscous fluxes; HLLC to Fc, viscous to Fv.
template <int LIM, int D, bool X>
__device__ __forceinline__ void face2(const Smem& s, int ca, int cb, V (&Fc)[4], V (&Fv)[4]) {
    using A = Ar<X>;
    constexpr int st = D == 0 ? 1 : LX;  // along the normal
    constexpr int tn = D == 0 ? LX : 1;  // along the face
    V pl[4], pr[4], wl[4], wr[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float* w = s.W[v];
        const V a = v2(w[ca - st], w[cb - st]);
        pl[v] = v2(w[ca], w[cb]);
        pr[v] = v2(w[ca + st], w[cb + st]);
        const V b = v2(w[ca + 2 * st], w[cb + 2 * st]);
        const V dc = A::sub(pr[v], pl[v]);
        const V sl = slope2<LIM, X>(A::sub(pl[v], a), dc);
        const V sr = slope2<LIM, X>(dc, A::sub(b, pr[v]));
        wl[v] = A::fma(sp(0.5f), sl, pl[v]);   // w + slope / 2
        wr[v] = A::fma(sp(-0.5f), sr, pr[v]);  // w - slope / 2
    }
    hllc2<D, X>(wl, wr, Fc);
    const V half = sp(0.5f);
    auto tangential = [&](const float* q) {  // the mean of the two cells' central differences along the face
        const V gl = A::mul(half, A::sub(v2(q[ca + tn], q[cb + tn]), v2(q[ca - tn], q[cb - tn])));
        const V gr = A::mul(half, A::sub(v2(q[ca + st + tn], q[cb + st + tn]), v2(q[ca + st - tn], q[cb + st - tn])));
        return A::mul(half, A::add(gl, gr));
    };
    visc2<D, X>(pl, pr, v2(s.T[ca], s.T[cb]), v2(s.T[ca + st], s.T[cb + st]), tangential(s.W[1]),
                tangential(s.W[2]), tangential(s.T), Fv);
}

template <int D, int stride>
__device__ __forceinline__ void store_face(float* out, int ia, int ib, const V (&Fc)[4], const V (&Fv)[4]) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        out[v * stride + ia] = Fc[v].x;
        out[v * stride + ib] = Fc[v].y;
        out[(4 + v) * stride + ia] = Fv[v].x;
        out[(4 + v) * stride + ib] = Fv[v].y;
    }
}

struct K {
    int nx, ny, walls, tiles_x;
    int64_t tiles;
    const float* U;
    // a y-slab of a larger grid: an edge whose bit is set in `edges` (1: below row 0, 2: above row ny - 1) is interior,
    // and its two rows of each field come from halo_lo / halo_hi, (4, 2, nx) each, instead of the boundary rule
    const float* halo_lo;
    const float* halo_hi;
    int edges;
    float* R;
    float* diag;
    double* det_sq64;
    uint32_t* ctrl;   // words 16: ~bits(min dt), 17: bits(max ws), 18..21: Σ R² (f32 atomics), kDone0: groups done
    float* part_dt;   // per tile
    float* part_ws;
    double* part_sq;  // [tiles][4]
    // the tiles in groups of kGroup consecutive ones: a completion count per group, and the group's combined partials
    int64_t groups;
    uint32_t* gdone;
    float* gpart_dt;
    float* gpart_ws;
    double* gpart_sq;  // [groups][4]
};

constexpr int kDtKey = 16, kWsBits = 17, kSq0 = 18;
constexpr int kGroup = kThreads;  // tiles per group: one partial per thread of the group's last block

__device__ __forceinline__ int wrapi(int k, int n) { return ((k % n) + n) % n; }

// dt and wave speed of one cell from its primitives (cell_diag, physics.hpp:196-202)
template <bool X>
__device__ __forceinline__ void cell_dt_ws(float rho, float u, float v, float p, float T, float& dt, float& ws) {
    if constexpr (X) {
        const float c = __fsqrt_rn(__fdiv_rn(__fmul_rn(kG, p), rho));
        const float ax = __fadd_rn(fabsf(u), c), ay = __fadd_rn(fabsf(v), c);
        const float nu = __fmul_rn(__fdiv_rn(kMu, rho), kNuMax);
        dt = __fdiv_rn(kCfl, __fadd_rn(__fadd_rn(ax, ay), __fmul_rn(4.0f, nu)));
        ws = ax > ay ? ax : ay;
    } else {
        const float c = sqrtf(kG * T);  // T = p / ρ
        const float ax = fabsf(u) + c, ay = fabsf(v) + c;
        const float nu = kMu * __frcp_rn(rho) * kNuMax;
        dt = kCfl / (ax + ay + 4.0f * nu);
        ws = fmaxf(ax, ay);
    }
}

template <int LIM, bool X>
__global__ void __launch_bounds__(kThreads, 4) k_ns_comp(K g) {
    using A = Ar<X>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& s = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tile = blockIdx.x;
    const int tx0 = (tile % g.tiles_x) * TX, ty0 = (tile / g.tiles_x) * TY;
    const int64_t plane = int64_t(g.nx) * g.ny;

    // 1. the tile and its halo, boundary rule on the fly, as primitives (tile_load + tile_boundary + to_prim). The fast
    // form has a thread issue the loads of all its cells (up to NL) before it converts any of them: one DRAM latency
    // per tile, not NL (0.505 -> 0.493 ms at 4096²). The reference-rounding form converts one cell at a time: its IEEE
    // divisions need the registers (0.72 ms the other way, against 0.69).
    if constexpr (!X) {
        constexpr int NL = (LC + kThreads - 1) / kThreads;
        float ld_r[NL], ld_mu[NL], ld_mv[NL], ld_E[NL];
        uint32_t flip = 0;  // bit q: cell q's momenta change sign (a wall's mirror image)
#pragma unroll
        for (int q = 0; q < NL; ++q) {
            const int idx = tid + q * kThreads;
            ld_r[q] = ld_mu[q] = ld_mv[q] = ld_E[q] = 0.0f;
            if (idx < LC) {
                const int lb = idx / LX, la = idx - lb * LX;
                const int j = ty0 - 2 + lb, i = tx0 - 2 + la;
                const int is = unsigned(i) < unsigned(g.nx) ? i : wrapi(i, g.nx);  // only halo columns wrap
                int js = j;
                const float* src = g.U;
                int64_t fs = plane;  // between the fields of src
                if (j < 0 || j >= g.ny) {
                    const bool lo = j < 0;
                    if (g.edges & (lo ? 1 : 2)) {  // a slab's interior edge: the neighbour's rows
                        src = lo ? g.halo_lo : g.halo_hi;
                        fs = 2 * int64_t(g.nx);
                        js = lo ? j + 2 : j - g.ny;
                    } else if (g.walls) {
                        js = lo ? -1 - j : 2 * g.ny - 1 - j;
                        flip |= 1u << q;
                    } else {
                        js = wrapi(j, g.ny);
                    }
                }
                const int64_t c = int64_t(js) * g.nx + is;
                ld_r[q] = __ldg(src + c);
                ld_mu[q] = __ldg(src + fs + c);
                ld_mv[q] = __ldg(src + 2 * fs + c);
                ld_E[q] = __ldg(src + 3 * fs + c);
            }
        }
#pragma unroll
        for (int q = 0; q < NL; ++q) {
            const int idx = tid + q * kThreads;
            if (idx >= LC) continue;
            const float r = ld_r[q];
            const bool neg = (flip >> q) & 1u;  // a sign flip: exact
            const float mu = neg ? -ld_mu[q] : ld_mu[q];
            const float mv = neg ? -ld_mv[q] : ld_mv[q];
            const float E = ld_E[q];
            const float ir = __frcp_rn(r);
            const float u = mu * ir, v = mv * ir;
            const float p = kGm1 * (E - 0.5f * r * (u * u + v * v));
            s.W[0][idx] = r;
            s.W[1][idx] = u;
            s.W[2][idx] = v;
            s.W[3][idx] = p;
            s.T[idx] = p * ir;
        }
    } else {
        for (int idx = tid; idx < LC; idx += kThreads) {
            const int lb = idx / LX, la = idx - lb * LX;
            const int j = ty0 - 2 + lb, i = tx0 - 2 + la;
            const int is = unsigned(i) < unsigned(g.nx) ? i : wrapi(i, g.nx);  // only halo columns wrap
            int js = j;
            float sg = 1.0f;
            const float* src = g.U;
            int64_t fs = plane;  // between the fields of src
            if (j < 0 || j >= g.ny) {
                const bool lo = j < 0;
                if (g.edges & (lo ? 1 : 2)) {  // a slab's interior edge: the neighbour's rows
                    src = lo ? g.halo_lo : g.halo_hi;
                    fs = 2 * int64_t(g.nx);
                    js = lo ? j + 2 : j - g.ny;
                } else if (g.walls) {
                    js = lo ? -1 - j : 2 * g.ny - 1 - j;
                    sg = -1.0f;
                } else {
                    js = wrapi(j, g.ny);
                }
            }
            const int64_t c = int64_t(js) * g.nx + is;
            const float r = __ldg(src + c);
            const float mu = __ldg(src + fs + c) * sg;  // a sign flip: exact
            const float mv = __ldg(src + 2 * fs + c) * sg;
            const float E = __ldg(src + 3 * fs + c);
            const float u = __fdiv_rn(mu, r), v = __fdiv_rn(mv, r);
            const float p =
                __fmul_rn(kGm1, __fsub_rn(E, __fmul_rn(__fmul_rn(0.5f, r), __fadd_rn(__fmul_rn(u, u), __fmul_rn(v, v)))));
            s.W[0][idx] = r;
            s.W[1][idx] = u;
            s.W[2][idx] = v;
            s.W[3][idx] = p;
            s.T[idx] = __fdiv_rn(p, r);
        }
    }
    __syncthreads();

    // 2. every face of the tile's cells, once, two per thread (tile_gradients, tile_reconstruct, tile_conv_flux,
    // tile_visc_flux). A warp takes one row of 32 faces for each lane of its pairs, so its shared-memory reads are
    // conflict-free. y-faces: face rows f = warp and f + 8 (face row f is the south face of tile row f; row 15 the
    // north face of row 14). x-faces: rows warp and warp + 8 (warps 0..6); warp 7 takes row 7 and, in its second
    // lanes, the 15 east faces of column 31. Every thread evaluates two y-faces and two x-faces: no warp waits for
    // another at the barrier, and each direction is one copy of the face code, so a face on the tile's north or
    // east edge, which the neighbouring tile evaluates too, gets the same bits from both.
    {
        V Fc[4], Fv[4];
        const int f = warp, k = lane;
        // y: between smem cells (f + 1, k + 2) and (f + 2, k + 2)
        face2<LIM, 1, X>(s, (f + 1) * LX + (k + 2), (f + 9) * LX + (k + 2), Fc, Fv);
        store_face<1, NYF>(&s.FY[0][0], f * TX + k, (f + 8) * TX + k, Fc, Fv);
        // x: the west face of tile cell (r, c) lies between smem cells (r + 2, c + 1) and (r + 2, c + 2)
        const bool east = warp == 7;
        const int rb = east ? (lane < TY ? lane : lane - TY) : f + 8, cb_ = east ? TX : k;
        face2<LIM, 0, X>(s, (f + 2) * LX + (k + 1), (rb + 2) * LX + (cb_ + 1), Fc, Fv);
        const int ia = f * (TX + 1) + k, ib = rb * (TX + 1) + cb_;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            s.FX[v][ia] = Fc[v].x;
            s.FX[4 + v][ia] = Fv[v].x;
        }
        if (!east || lane < TY) {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                s.FX[v][ib] = Fc[v].y;
                s.FX[4 + v][ib] = Fv[v].y;
            }
        }
    }
    __syncthreads();

    // 3. R = -div F_conv + div F_visc per cell (cell_divergence: conv, then visc added), two cells per thread (rows r and
    // r + 8 of column k; warp 7 has row 7 only), and the per-cell diagnostics
    float dtmin = 3.0e38f, wsmax = 0.0f;
    double sqd[4] = {0.0, 0.0, 0.0, 0.0};
    {
        const int r = warp, k = lane;
        const int r1 = warp < 7 ? r + 8 : r;  // warp 7: the second lane repeats the first (not stored)
        const int j0 = ty0 + r, j1 = ty0 + r1, i = tx0 + k;
        const bool in0 = j0 < g.ny && i < g.nx, in1 = warp < 7 && j1 < g.ny && i < g.nx;
        const int xw0 = r * (TX + 1) + k, xw1 = r1 * (TX + 1) + k;
        const int ys0 = r * TX + k, ys1 = r1 * TX + k;
        const int64_t o0 = int64_t(j0) * g.nx + i, o1 = int64_t(j1) * g.nx + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float* fx = s.FX[v];
            const float* fy = s.FY[v];
            const float* gx = s.FX[4 + v];
            const float* gy = s.FY[4 + v];
            const V divc = A::add(A::sub(v2(fx[xw0 + 1], fx[xw1 + 1]), v2(fx[xw0], fx[xw1])),
                                  A::sub(v2(fy[ys0 + TX], fy[ys1 + TX]), v2(fy[ys0], fy[ys1])));
            const V divv = A::add(A::sub(v2(gx[xw0 + 1], gx[xw1 + 1]), v2(gx[xw0], gx[xw1])),
                                  A::sub(v2(gy[ys0 + TX], gy[ys1 + TX]), v2(gy[ys0], gy[ys1])));
            const V rv = A::sub(divv, divc);  // -divc + divv: the same bits
            if (in0) {
                g.R[v * plane + o0] = rv.x;
                sqd[v] = __fma_rn(double(rv.x), double(rv.x), sqd[v]);
            }
            if (in1) {
                g.R[v * plane + o1] = rv.y;
                sqd[v] = __fma_rn(double(rv.y), double(rv.y), sqd[v]);
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            if (h == 0 ? !in0 : !in1) continue;
            const int c = ((h == 0 ? r : r1) + 2) * LX + (k + 2);
            float dt, ws;
            cell_dt_ws<X>(s.W[0][c], s.W[1][c], s.W[2][c], s.W[3][c], s.T[c], dt, ws);
            dtmin = fminf(dtmin, dt);
            wsmax = fmaxf(wsmax, ws);
        }
    }

    // 4. the tile's reductions (fixed order: xor tree in the warp, warps in order). The tile's Σ R² is summed once, in
    // f64: the deterministic path keeps it, the atomic path adds it rounded to f32 (the reference's atomic stage adds
    // each tile's f32 group sum; either way the atomic total depends on the order the tiles finish in).
    // The deterministic path then combines the tiles in two levels, each in a fixed order: the last tile to finish in
    // each group of kGroup consecutive tiles combines the group's tile partials (one per thread), and the last group
    // the group partials. One block reading every tile's partials at the end held the launch's tail: 44 µs of the
    // 0.492 ms at 4096² (35,072 tiles, 137 dependent rounds of L2 loads per thread).
    __shared__ float r_dt[kThreads / 32], r_ws[kThreads / 32];
    __shared__ double r_sqd[kThreads / 32][4];
    __shared__ int s_last;
    // min dt, max wave speed and Σ R² over the block's threads (the group and final levels): an xor tree in each warp,
    // then warps 0..7 in order by thread 0, which holds the block's values afterwards
    auto block_combine = [&](float& dm, float& wm, double (&sd)[4]) {
#pragma unroll
        for (int off = 16; off >= 1; off >>= 1) {
            dm = fminf(dm, __shfl_xor_sync(0xffffffffu, dm, off));
            wm = fmaxf(wm, __shfl_xor_sync(0xffffffffu, wm, off));
#pragma unroll
            for (int v = 0; v < 4; ++v) sd[v] += __shfl_xor_sync(0xffffffffu, sd[v], off);
        }
        __syncthreads();  // r_* are free
        if (lane == 0) {
            r_dt[warp] = dm;
            r_ws[warp] = wm;
#pragma unroll
            for (int v = 0; v < 4; ++v) r_sqd[warp][v] = sd[v];
        }
        __syncthreads();
        if (tid == 0) {
            dm = r_dt[0];
            wm = r_ws[0];
#pragma unroll
            for (int v = 0; v < 4; ++v) sd[v] = r_sqd[0][v];
            for (int w = 1; w < kThreads / 32; ++w) {
                dm = fminf(dm, r_dt[w]);
                wm = fmaxf(wm, r_ws[w]);
#pragma unroll
                for (int v = 0; v < 4; ++v) sd[v] += r_sqd[w][v];
            }
        }
    };
    // The tile's own values: every thread writes its min dt, max wave speed and four Σ R² into the tile's shared
    // memory (free once every warp is done with phase 3), and warp 0 alone combines them: lane l takes threads l,
    // l + 32, ..., l + 224 in order, then an xor tree over the lanes. The other warps skip the tree's shuffles (about
    // 80 instructions a thread, 6 % of a tile's).
    {
        __syncthreads();  // phase 3's reads of the tile's shared memory are over
        float* const mm = s.T;                                       // [2][kThreads] (T holds LC >= 512 floats)
        double* const sq = reinterpret_cast<double*>(&s.FX[0][0]);  // [4][kThreads] (FX starts 8-byte aligned)
        mm[tid] = dtmin;
        mm[kThreads + tid] = wsmax;
#pragma unroll
        for (int v = 0; v < 4; ++v) sq[v * kThreads + tid] = sqd[v];
        __syncthreads();
        if (warp == 0) {
            dtmin = mm[lane];
            wsmax = mm[kThreads + lane];
#pragma unroll
            for (int v = 0; v < 4; ++v) sqd[v] = sq[v * kThreads + lane];
#pragma unroll
            for (int w = 1; w < kThreads / 32; ++w) {
                dtmin = fminf(dtmin, mm[w * 32 + lane]);
                wsmax = fmaxf(wsmax, mm[kThreads + w * 32 + lane]);
#pragma unroll
                for (int v = 0; v < 4; ++v) sqd[v] += sq[v * kThreads + w * 32 + lane];
            }
#pragma unroll
            for (int off = 16; off >= 1; off >>= 1) {
                dtmin = fminf(dtmin, __shfl_xor_sync(0xffffffffu, dtmin, off));
                wsmax = fmaxf(wsmax, __shfl_xor_sync(0xffffffffu, wsmax, off));
#pragma unroll
                for (int v = 0; v < 4; ++v) sqd[v] += __shfl_xor_sync(0xffffffffu, sqd[v], off);
            }
        }
    }
    const int64_t grp = tile / kGroup;
    if (tid == 0) {
        g.part_dt[tile] = dtmin;
        g.part_ws[tile] = wsmax;
#pragma unroll
        for (int v = 0; v < 4; ++v) g.part_sq[int64_t(tile) * 4 + v] = sqd[v];
        // the atomic path: positive floats order like their bit patterns
        atomicMax(g.ctrl + kDtKey, 0xffffffffu - __float_as_uint(dtmin));
        atomicMax(g.ctrl + kWsBits, __float_as_uint(wsmax));
#pragma unroll
        for (int v = 0; v < 4; ++v) atomicAdd(reinterpret_cast<float*>(g.ctrl + kSq0 + v), float(sqd[v]));
        __threadfence();
        const int64_t gsize = g.tiles - grp * kGroup < kGroup ? g.tiles - grp * kGroup : kGroup;
        s_last = atomicAdd(g.gdone + grp, 1u) == uint32_t(gsize - 1);
        if (s_last) __threadfence();  // for the whole block: the barrier orders the others' loads after it
    }
    __syncthreads();
    if (!s_last) return;

    // 5. the last tile of its group: the group's tile partials in tile order (thread t: tile grp·kGroup + t). One
    // thread fences (above), not every thread: a warp's fence would first wait for its residual stores to drain.
    {
        const int64_t t = grp * kGroup + tid;
        float dm = 3.0e38f, wm = 0.0f;
        double sd[4] = {0.0, 0.0, 0.0, 0.0};
        if (t < g.tiles) {
            dm = __ldcg(g.part_dt + t);
            wm = __ldcg(g.part_ws + t);
#pragma unroll
            for (int v = 0; v < 4; ++v) sd[v] = __ldcg(g.part_sq + t * 4 + v);
        }
        block_combine(dm, wm, sd);
        if (tid == 0) {
            g.gpart_dt[grp] = dm;
            g.gpart_ws[grp] = wm;
#pragma unroll
            for (int v = 0; v < 4; ++v) g.gpart_sq[grp * 4 + v] = sd[v];
            __threadfence();
            s_last = atomicAdd(g.ctrl + kDone0, 1u) == uint32_t(g.groups - 1);
            if (s_last) __threadfence();
        }
        __syncthreads();
    }
    if (!s_last) return;

    // 6. the last group: the group partials in group order (thread t: groups t, t + 256, ...), and the error stage
    float dm = 3.0e38f, wm = 0.0f;
    double sd[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t q = tid; q < g.groups; q += kThreads) {
        dm = fminf(dm, __ldcg(g.gpart_dt + q));
        wm = fmaxf(wm, __ldcg(g.gpart_ws + q));
#pragma unroll
        for (int v = 0; v < 4; ++v) sd[v] += __ldcg(g.gpart_sq + q * 4 + v);
    }
    block_combine(dm, wm, sd);
    if (tid == 0) {
        const float DetDt = dm, DetWs = wm;
        const double* DetSq = sd;
        const float Dt = __uint_as_float(0xffffffffu - ld_volatile(g.ctrl + kDtKey));
        const float Ws = __uint_as_float(ld_volatile(g.ctrl + kWsBits));
        float Sq[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) Sq[v] = __uint_as_float(ld_volatile(g.ctrl + kSq0 + v));
        float* D = g.diag;
        D[0] = Dt;
        D[1] = Ws;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            D[2 + v] = Sq[v];
            D[6 + v] = float(DetSq[v]);
            if (g.det_sq64) g.det_sq64[v] = DetSq[v];
        }
        D[10] = DetDt;
        D[11] = DetWs;
        D[12] = Dt - DetDt;
        D[13] = Ws - DetWs;
#pragma unroll
        for (int v = 0; v < 4; ++v) D[14 + v] = Sq[v] - float(DetSq[v]);
    }
}

// The initial field (physics.hpp:203-215, make_init main.cpp:100-112).
__global__ void k_init_cons(float* U, int nx, int ny, float amp) {
    const int64_t n = int64_t(nx) * ny;
    const float k = float(2.0 * 3.14159265358979323846 / 32.0);
    for (int64_t c = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; c < n; c += int64_t(gridDim.x) * blockDim.x) {
        const int j = int(c / nx), i = int(c - int64_t(j) * nx);
        const float x = float(i) + 0.5f, y = float(j) + 0.5f;
        const float sx = sinf(k * x), cx = cosf(k * x), sy = sinf(k * y), cy = cosf(k * y);
        const float r = 1.0f + 0.1f * amp * sx * sy;
        const float u = 0.3f + 0.05f * amp * cx * sy;
        const float v = 0.2f + 0.05f * amp * sx * cy;
        const float p = 1.0f + 0.05f * amp * cx * cy;
        U[c] = r;
        U[n + c] = r * u;
        U[2 * n + c] = r * v;
        U[3 * n + c] = p / (kG - 1.0f) + 0.5f * r * (u * u + v * v);
    }
}

}  // namespace nsc
}  // namespace cspb

using namespace cspb;
using cspb_host::align_up;
using cspb_host::aligned;

namespace {

struct NscLayout {
    int tiles_x = 0;
    int64_t tiles = 0, groups = 0;
    size_t off_gdone = 0, zero_bytes = 0, off_dt = 0, off_ws = 0, off_sq = 0, off_gdt = 0, off_gws = 0, off_gsq = 0,
           total = 0;
};

// [control block][group counters] (zeroed before each launch), then the tile and group partials
NscLayout nsc_layout(int nx, int ny) {
    NscLayout L;
    L.tiles_x = (nx + nsc::TX - 1) / nsc::TX;
    L.tiles = int64_t(L.tiles_x) * ((ny + nsc::TY - 1) / nsc::TY);
    L.groups = (L.tiles + nsc::kGroup - 1) / nsc::kGroup;
    size_t o = kCtrlBytes;
    L.off_gdone = o;
    o = align_up(o + size_t(L.groups) * 4, 256);
    L.zero_bytes = o;
    L.off_dt = o;
    o = align_up(o + size_t(L.tiles) * 4, 256);
    L.off_ws = o;
    o = align_up(o + size_t(L.tiles) * 4, 256);
    L.off_sq = o;
    o = align_up(o + size_t(L.tiles) * 32, 256);
    L.off_gdt = o;
    o = align_up(o + size_t(L.groups) * 4, 256);
    L.off_gws = o;
    o = align_up(o + size_t(L.groups) * 4, 256);
    L.off_gsq = o;
    o = align_up(o + size_t(L.groups) * 32, 256);
    L.total = o;
    return L;
}

}  // namespace

extern "C" {

size_t cspb_ns_comp_workspace_bytes(int32_t nx, int32_t ny) {
    if (nx < 4 || ny < 4) return 0;
    return nsc_layout(nx, ny).total;
}

}  // extern "C"

namespace {

// One launch over ny × nx cells (a whole grid, or a slab when edges != 0).
int launch_ns_comp(int nx, int ny, int limiter, int walls, int flags, const float* U, const float* halo_lo,
                   const float* halo_hi, int edges, float* R, float* diag, double* det_sq64, void* workspace,
                   size_t workspace_bytes, cudaStream_t st) {
    if (limiter != 0 && limiter != 1) return CSPB_ERR_UNSUPPORTED;
    if (walls != 0 && walls != 1) return CSPB_ERR_ARGUMENT;
    if ((flags & ~CSPB_NS_REFERENCE_ROUNDING) != 0) return CSPB_ERR_ARGUMENT;
    if (int64_t(nx) * ny > (int64_t(1) << 31)) return CSPB_ERR_ARGUMENT;
    const NscLayout L = nsc_layout(nx, ny);
    if (!workspace || !aligned(workspace, 256) || workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    if (L.tiles > 0x7fffffff) return CSPB_ERR_ARGUMENT;
    char* ws = static_cast<char*>(workspace);
    if (cudaMemsetAsync(ws, 0, L.zero_bytes, st) != cudaSuccess) return CSPB_ERR_CUDA;
    nsc::K g{};
    g.nx = nx;
    g.ny = ny;
    g.walls = walls;
    g.tiles_x = L.tiles_x;
    g.tiles = L.tiles;
    g.U = U;
    g.halo_lo = halo_lo;
    g.halo_hi = halo_hi;
    g.edges = edges;
    g.R = R;
    g.diag = diag;
    g.det_sq64 = det_sq64;
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    g.part_dt = reinterpret_cast<float*>(ws + L.off_dt);
    g.part_ws = reinterpret_cast<float*>(ws + L.off_ws);
    g.part_sq = reinterpret_cast<double*>(ws + L.off_sq);
    g.groups = L.groups;
    g.gdone = reinterpret_cast<uint32_t*>(ws + L.off_gdone);
    g.gpart_dt = reinterpret_cast<float*>(ws + L.off_gdt);
    g.gpart_ws = reinterpret_cast<float*>(ws + L.off_gws);
    g.gpart_sq = reinterpret_cast<double*>(ws + L.off_gsq);
    const size_t smem = sizeof(nsc::Smem);
    const bool exact = (flags & CSPB_NS_REFERENCE_ROUNDING) != 0;
    auto kern = limiter == 0 ? (exact ? nsc::k_ns_comp<0, true> : nsc::k_ns_comp<0, false>)
                             : (exact ? nsc::k_ns_comp<1, true> : nsc::k_ns_comp<1, false>);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return CSPB_ERR_CUDA;
    kern<<<unsigned(L.tiles), nsc::kThreads, smem, st>>>(g);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

}  // namespace

extern "C" {

int cspb_ns_compressible(const cspb_ns_comp_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (d->nx < 4 || d->ny < 4 || !d->U || !d->R || !d->diag) return CSPB_ERR_ARGUMENT;
    if (d->reserved != 0) return CSPB_ERR_ARGUMENT;
    return launch_ns_comp(d->nx, d->ny, d->limiter, d->walls, d->flags, d->U, nullptr, nullptr, 0, d->R, d->diag,
                          d->det_sq64, d->workspace, d->workspace_bytes, static_cast<cudaStream_t>(stream));
}

size_t cspb_ns_comp_slab_workspace_bytes(int32_t nx, int32_t rows) {
    if (nx < 4 || rows < 2) return 0;
    return nsc_layout(nx, rows).total;
}

int cspb_ns_comp_slab(const cspb_ns_comp_slab_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (d->nx < 4 || d->rows < 2 || !d->U || !d->R || !d->diag) return CSPB_ERR_ARGUMENT;
    if ((d->edges & ~3) != 0 || ((d->edges & 1) && !d->halo_lo) || ((d->edges & 2) && !d->halo_hi))
        return CSPB_ERR_ARGUMENT;
    return launch_ns_comp(d->nx, d->rows, d->limiter, d->walls, d->flags, d->U, d->halo_lo, d->halo_hi, d->edges,
                          d->R, d->diag, d->det_sq64, d->workspace, d->workspace_bytes,
                          static_cast<cudaStream_t>(stream));
}

int cspb_ns_init_cons(float* U, int32_t nx, int32_t ny, float amp, void* stream) {
    if (!U || nx < 1 || ny < 1) return CSPB_ERR_ARGUMENT;
    const int64_t n = int64_t(nx) * ny;
    int64_t blocks = (n + 255) / 256;
    if (blocks > 65535) blocks = 65535;
    nsc::k_init_cons<<<unsigned(blocks), 256, 0, static_cast<cudaStream_t>(stream)>>>(U, nx, ny, amp);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

}  // extern "C"
