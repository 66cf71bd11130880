// ns_comp.cu — the reference's compressible Navier-Stokes residual and its diagnostics in ONE kernel.
//
// Reproduces examples/ns-residual: the physics of physics.hpp (to_prim :86-94, grad_cell :97-104, HLLC :109-152,
// visc_flux :157-192, cell_diag :196-202, MinMod / VanLeer :62-80), the tile stages of tile.hpp:39-229, and the
// diagnostics of components.hpp:393-628 (atomic min dt / max wave speed / Σ R², their deterministic fixed-order
// counterparts, and the error stage atomic − deterministic).
//
// The reference's fused group (systems.hpp:88-140) and its hand-written kernel (handwritten.hpp:51-191) write the four
// face-flux arrays to global memory and wait on neighbour tiles before the divergence (≈1 GiB round trip at 4096²).
// Here a block owns a 32×16 tile and keeps everything on chip: it loads the tile with a 2-cell halo (boundary rule
// applied on the fly), forms primitives, cell gradients and MUSCL slopes in shared memory, evaluates every face of its
// cells once — the faces on the tile's east and north edges are evaluated by both neighbouring tiles, with identical
// arithmetic, so R is independent of the tiling — and writes R. HBM traffic is one read of U and one write of R
// (32 B/cell); the halo re-reads are L2 hits.
//
// Diagnostics: per tile, min dt, max wave speed and Σ R² (f32 for the atomic path, f64 for the deterministic one) in a
// fixed order; atomics for the atomic path (integer max on the bit patterns of positive floats for min / max, float
// add for the sums); per-tile partials, and the last block to finish reduces them in tile order (min / max exactly,
// sums in f64) and writes the error stage. Deterministic results are bit-identical on every run.
#include "common.cuh"

namespace cspb {
namespace nsc {

constexpr int TX = 32, TY = 16;              // tile of cells
constexpr int LX = TX + 4, LY = TY + 4;      // with the 2-cell halo
constexpr int LC = LX * LY;                  // 720
constexpr int NXF = (TX + 1) * TY;           // x-faces of the tile's rows
constexpr int NYF = TX * (TY + 1);           // y-faces of the tile's columns
constexpr int kThreads = 256;

constexpr float kG = 1.4f, kMu = 0.01f, kPr = 0.72f, kCfl = 0.5f;

// The tile's state in shared memory: primitives and temperature of the tile with its 2-cell halo, and both fluxes of
// every face. A face forms the gradients and limited slopes of its two cells from W and T itself, with the formulas
// a per-cell table would hold (the same bits): a table of both for the 612 cells [-1, T] took 34 KB more, which left
// room for 2 tiles per SM instead of 4.
struct Smem {
    float W[4][LC];  // primitives ρ u v p
    float T[LC];     // p / ρ
    float FX[8][NXF];  // HLLC 0..3, viscous 4..7
    float FY[8][NYF];
};

__device__ __forceinline__ float fmn(float a, float b) { return a < b ? a : b; }
__device__ __forceinline__ float fmx(float a, float b) { return a > b ? a : b; }

template <int LIM>
__device__ __forceinline__ float slope(float a, float b) {
    if (LIM == 0) {
        if (a * b <= 0.0f) return 0.0f;
        return a > 0.0f ? fmn(a, b) : fmx(a, b);
    } else {
        const float ab = a * b;
        if (ab <= 0.0f) return 0.0f;
        return 2.0f * ab / (a + b);
    }
}

// 1 / (γ - 1), rounded once
constexpr float kInvGm1 = 1.0f / (kG - 1.0f);

// HLLC with Davis speeds; D = 0 normal x, D = 1 normal y; L / R primitives (ρ, u, v, p). The divisions by ρ of a side
// are products with its reciprocal, p / (γ - 1) a product with 1 / (γ - 1). The face's reciprocals, square roots and
// divisions use the hardware's approximate forms (__fdividef, rsqrtf: about 2 ulp): at 4096² they took the kernel
// from 0.709 to 0.657 ms, and the residual's relative L2 error against the f64 oracle from 4.4e-6 to 4.7e-6 (the f32
// storage of U dominates it; the reference's bound is 1e-4). The per-cell phases, and so the diagnostics, keep the
// correctly rounded forms.
template <int D>
__device__ __forceinline__ void hllc(const float (&L)[4], const float (&R)[4], float (&F)[4]) {
    const float rl = L[0], rr = R[0], pl = L[3], pr = R[3];
    const float unl = L[1 + D], utl = L[2 - D];
    const float unr = R[1 + D], utr = R[2 - D];
    const float irl = __fdividef(1.0f, rl), irr = __fdividef(1.0f, rr);
    const float gl = kG * pl * irl, gr = kG * pr * irr;
    const float cl = gl > 0.0f ? gl * rsqrtf(gl) : 0.0f, cr = gr > 0.0f ? gr * rsqrtf(gr) : 0.0f;
    const float El = pl * kInvGm1 + 0.5f * rl * (unl * unl + utl * utl);
    const float Er = pr * kInvGm1 + 0.5f * rr * (unr * unr + utr * utr);
    const float sl = fmn(unl - cl, unr - cr);
    const float sr = fmx(unl + cl, unr + cr);
    const float sm = __fdividef(pr - pl + rl * unl * (sl - unl) - rr * unr * (sr - unr), rl * (sl - unl) - rr * (sr - unr));
    float f0, f1, f2, f3;
    if (sl >= 0.0f) {
        f0 = rl * unl; f1 = rl * unl * unl + pl; f2 = rl * unl * utl; f3 = (El + pl) * unl;
    } else if (sr <= 0.0f) {
        f0 = rr * unr; f1 = rr * unr * unr + pr; f2 = rr * unr * utr; f3 = (Er + pr) * unr;
    } else {
        const bool left = sm >= 0.0f;
        const float r = left ? rl : rr, un = left ? unl : unr, ut = left ? utl : utr, p = left ? pl : pr;
        const float E = left ? El : Er, s = left ? sl : sr, ir = left ? irl : irr;
        const float a = s - un;
        const float k = __fdividef(r * a, s - sm);
        const float Es = k * (E * ir + (sm - un) * (sm + __fdividef(p * ir, a)));
        f0 = r * un + s * (k - r);
        f1 = r * un * un + p + s * (k * sm - r * un);
        f2 = r * un * ut + s * (k * ut - r * ut);
        f3 = (E + p) * un + s * (Es - E);
    }
    F[0] = f0;
    F[1 + D] = f1;
    F[2 - D] = f2;
    F[3] = f3;
}

// The viscous flux through a face of normal D: the normal derivatives are the differences of the two cells; the
// tangential ones (ut_u, ut_v, ut_T) the means of the two cells' central differences.
template <int D>
__device__ __forceinline__ void visc(const float (&L)[4], const float (&R)[4], float TL, float TR, float du_t,
                                     float dv_t, float dT_t, float (&F)[4]) {
    const float uf = 0.5f * (L[1] + R[1]), vf = 0.5f * (L[2] + R[2]);
    float ux, uy, vx, vy, Tx, Ty;
    if (D == 0) {
        ux = R[1] - L[1]; vx = R[2] - L[2]; Tx = TR - TL;
        uy = du_t; vy = dv_t; Ty = dT_t;
    } else {
        uy = R[1] - L[1]; vy = R[2] - L[2]; Ty = TR - TL;
        ux = du_t; vx = dv_t; Tx = dT_t;
    }
    const float mu = kMu;
    const float k = mu * kG / ((kG - 1.0f) * kPr);
    const float dv = ux + vy;
    const float txx = mu * (2.0f * ux - 2.0f / 3.0f * dv);
    const float tyy = mu * (2.0f * vy - 2.0f / 3.0f * dv);
    const float txy = mu * (uy + vx);
    F[0] = 0.0f;
    if (D == 0) {
        F[1] = txx; F[2] = txy; F[3] = uf * txx + vf * txy + k * Tx;
    } else {
        F[1] = txy; F[2] = tyy; F[3] = uf * txy + vf * tyy + k * Ty;
    }
}

// One face of normal D between cells cl and cl + st (st the neighbour along the normal): the limited slopes of both
// cells along the normal, the reconstructed states, the HLLC flux, the tangential gradients of both cells and the
// viscous flux; the 8 fluxes go to out[v * stride] (HLLC 0..3, viscous 4..7).
template <int LIM, int D, int stride>
__device__ __forceinline__ void face(const Smem& s, int cl, float* out) {
    constexpr int st = D == 0 ? 1 : LX;  // along the normal
    constexpr int tn = D == 0 ? LX : 1;  // along the face
    const int cr = cl + st;
    float pl[4], pr[4], wl[4], wr[4], Fc[4], Fv[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const float a = s.W[v][cl - st], b = s.W[v][cr + st];
        pl[v] = s.W[v][cl];
        pr[v] = s.W[v][cr];
        const float sl = slope<LIM>(pl[v] - a, pr[v] - pl[v]);
        const float sr = slope<LIM>(pr[v] - pl[v], b - pr[v]);
        wl[v] = pl[v] + 0.5f * sl;
        wr[v] = pr[v] - 0.5f * sr;
    }
    hllc<D>(wl, wr, Fc);
    auto tangential = [&](const float* q) {  // the mean of the two cells' central differences along the face
        return 0.5f * (0.5f * (q[cl + tn] - q[cl - tn]) + 0.5f * (q[cr + tn] - q[cr - tn]));
    };
    visc<D>(pl, pr, s.T[cl], s.T[cr], tangential(s.W[1]), tangential(s.W[2]), tangential(s.T), Fv);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        out[v * stride] = Fc[v];
        out[(4 + v) * stride] = Fv[v];
    }
}

struct K {
    int nx, ny, walls, tiles_x;
    int64_t tiles;
    const float* U;
    float* R;
    float* diag;
    double* det_sq64;
    uint32_t* ctrl;   // words 16: ~bits(min dt), 17: bits(max ws), 18..21: Σ R² (f32 atomics), kDone0: tiles done
    float* part_dt;
    float* part_ws;
    double* part_sq;  // [tiles][4]
};

constexpr int kDtKey = 16, kWsBits = 17, kSq0 = 18;

__device__ __forceinline__ int wrapi(int k, int n) { return ((k % n) + n) % n; }

template <int LIM>
__global__ void __launch_bounds__(kThreads, 4) k_ns_comp(K g) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    Smem& s = *reinterpret_cast<Smem*>(smem_raw);
    const int tid = threadIdx.x;
    const int tile = blockIdx.x;
    const int tx0 = (tile % g.tiles_x) * TX, ty0 = (tile / g.tiles_x) * TY;
    const int64_t plane = int64_t(g.nx) * g.ny;

    // 1. the tile and its halo, boundary rule on the fly, as primitives (tile_load + tile_boundary + to_prim)
    for (int idx = tid; idx < LC; idx += kThreads) {
        const int lb = idx / LX, la = idx - lb * LX;
        const int j = ty0 - 2 + lb, i = tx0 - 2 + la;
        const int is = unsigned(i) < unsigned(g.nx) ? i : wrapi(i, g.nx);  // only halo columns wrap
        int js = j;
        float sg = 1.0f;
        if (j < 0 || j >= g.ny) {
            if (g.walls) {
                js = j < 0 ? -1 - j : 2 * g.ny - 1 - j;
                sg = -1.0f;
            } else {
                js = wrapi(j, g.ny);
            }
        }
        const int64_t c = int64_t(js) * g.nx + is;
        const float r = __ldg(g.U + c);
        const float mu = __ldg(g.U + plane + c) * sg;
        const float mv = __ldg(g.U + 2 * plane + c) * sg;
        const float E = __ldg(g.U + 3 * plane + c);
        const float ir = __frcp_rn(r);
        const float u = mu * ir, v = mv * ir;
        const float p = (kG - 1.0f) * (E - 0.5f * r * (u * u + v * v));
        s.W[0][idx] = r;
        s.W[1][idx] = u;
        s.W[2][idx] = v;
        s.W[3][idx] = p;
        s.T[idx] = p * ir;
    }
    __syncthreads();

    // 2. every face of the tile's cells, once (tile_gradients, tile_reconstruct, tile_conv_flux, tile_visc_flux).
    // Work items in warp-uniform runs: the 17 rows of y-faces, the 16 rows of x-faces west of each tile cell (a warp
    // per row, so the reads are conflict-free), then the 16 x-faces on the tile's east edge.
    for (int f = tid; f < NXF + NYF; f += kThreads) {
        if (f < NYF) {
            const int r = f / TX, k = f - r * TX;  // between tile cells (r-1, k) and (r, k)
            face<LIM, 1, NYF>(s, (r + 1) * LX + (k + 2), &s.FY[0][f]);
        } else {
            int r, k;  // between tile cells (r, k-1) and (r, k)
            const int q = f - NYF;
            if (q < TY * TX) {
                r = q / TX;
                k = q - r * TX;
            } else {
                r = q - TY * TX;
                k = TX;
            }
            face<LIM, 0, NXF>(s, (r + 2) * LX + (k + 1), &s.FX[0][r * (TX + 1) + k]);
        }
    }
    __syncthreads();

    // 3. R = -div F_conv + div F_visc per cell (cell_divergence), and the per-cell diagnostics
    float dtmin = 3.0e38f, wsmax = 0.0f;
    float sqf[4] = {0.f, 0.f, 0.f, 0.f};
    double sqd[4] = {0.0, 0.0, 0.0, 0.0};
    for (int idx = tid; idx < TX * TY; idx += kThreads) {
        const int r = idx / TX, k = idx - r * TX;
        const int j = ty0 + r, i = tx0 + k;
        if (j >= g.ny || i >= g.nx) continue;
        const int xw = r * (TX + 1) + k, xe = xw + 1, ys = r * TX + k, yn = ys + TX;
        const int64_t o = int64_t(j) * g.nx + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float divc = (s.FX[v][xe] - s.FX[v][xw]) + (s.FY[v][yn] - s.FY[v][ys]);
            const float divv = (s.FX[4 + v][xe] - s.FX[4 + v][xw]) + (s.FY[4 + v][yn] - s.FY[4 + v][ys]);
            const float rv = -divc + divv;
            g.R[v * plane + o] = rv;
            sqf[v] += rv * rv;
            sqd[v] = __fma_rn(double(rv), double(rv), sqd[v]);
        }
        const int c = (r + 2) * LX + (k + 2);
        const float rho = s.W[0][c], u = s.W[1][c], vv = s.W[2][c];
        const float cs = sqrtf(kG * s.T[c]);  // T = p / ρ
        const float ax = fabsf(u) + cs, ay = fabsf(vv) + cs;
        const float nu = kMu * __frcp_rn(rho) * fmx(4.0f / 3.0f, kG / kPr);
        const float dt = kCfl / (ax + ay + 4.0f * nu);
        const float ws = fmx(ax, ay);
        dtmin = fmn(dtmin, dt);
        wsmax = fmx(wsmax, ws);
    }

    // 4. the tile's reductions (fixed order: xor tree in the warp, warps in order)
    __shared__ float r_dt[kThreads / 32], r_ws[kThreads / 32], r_sqf[kThreads / 32][4];
    __shared__ double r_sqd[kThreads / 32][4];
    __shared__ int s_last;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        dtmin = fmn(dtmin, __shfl_xor_sync(0xffffffffu, dtmin, off));
        wsmax = fmx(wsmax, __shfl_xor_sync(0xffffffffu, wsmax, off));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            sqf[v] += __shfl_xor_sync(0xffffffffu, sqf[v], off);
            sqd[v] += __shfl_xor_sync(0xffffffffu, sqd[v], off);
        }
    }
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) {
        r_dt[warp] = dtmin;
        r_ws[warp] = wsmax;
#pragma unroll
        for (int v = 0; v < 4; ++v) { r_sqf[warp][v] = sqf[v]; r_sqd[warp][v] = sqd[v]; }
    }
    __syncthreads();
    if (tid == 0) {
        float dm = r_dt[0], wm = r_ws[0], sf[4];
        double sd[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) { sf[v] = r_sqf[0][v]; sd[v] = r_sqd[0][v]; }
        for (int w = 1; w < kThreads / 32; ++w) {
            dm = fmn(dm, r_dt[w]);
            wm = fmx(wm, r_ws[w]);
#pragma unroll
            for (int v = 0; v < 4; ++v) { sf[v] += r_sqf[w][v]; sd[v] += r_sqd[w][v]; }
        }
        g.part_dt[tile] = dm;
        g.part_ws[tile] = wm;
#pragma unroll
        for (int v = 0; v < 4; ++v) g.part_sq[int64_t(tile) * 4 + v] = sd[v];
        // the atomic path: positive floats order like their bit patterns
        atomicMax(g.ctrl + kDtKey, 0xffffffffu - __float_as_uint(dm));
        atomicMax(g.ctrl + kWsBits, __float_as_uint(wm));
#pragma unroll
        for (int v = 0; v < 4; ++v) atomicAdd(reinterpret_cast<float*>(g.ctrl + kSq0 + v), sf[v]);
        __threadfence();
        s_last = atomicAdd(g.ctrl + kDone0, 1u) == uint32_t(g.tiles - 1);
    }
    __syncthreads();
    if (!s_last) return;

    // 6. the last tile: deterministic reductions of the per-tile partials in tile order, and the error stage
    __threadfence();
    float dm = 3.0e38f, wm = 0.0f;
    double sd[4] = {0.0, 0.0, 0.0, 0.0};
    for (int64_t t = tid; t < g.tiles; t += kThreads) {
        dm = fmn(dm, __ldcg(g.part_dt + t));
        wm = fmx(wm, __ldcg(g.part_ws + t));
#pragma unroll
        for (int v = 0; v < 4; ++v) sd[v] += __ldcg(g.part_sq + t * 4 + v);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        dm = fmn(dm, __shfl_xor_sync(0xffffffffu, dm, off));
        wm = fmx(wm, __shfl_xor_sync(0xffffffffu, wm, off));
#pragma unroll
        for (int v = 0; v < 4; ++v) sd[v] += __shfl_xor_sync(0xffffffffu, sd[v], off);
    }
    __syncthreads();
    if (lane == 0) {
        r_dt[warp] = dm;
        r_ws[warp] = wm;
#pragma unroll
        for (int v = 0; v < 4; ++v) r_sqd[warp][v] = sd[v];
    }
    __syncthreads();
    if (tid == 0) {
        float DetDt = r_dt[0], DetWs = r_ws[0];
        double DetSq[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) DetSq[v] = r_sqd[0][v];
        for (int w = 1; w < kThreads / 32; ++w) {
            DetDt = fmn(DetDt, r_dt[w]);
            DetWs = fmx(DetWs, r_ws[w]);
#pragma unroll
            for (int v = 0; v < 4; ++v) DetSq[v] += r_sqd[w][v];
        }
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
    int64_t tiles = 0;
    size_t off_dt = 0, off_ws = 0, off_sq = 0, total = 0;
};

NscLayout nsc_layout(int nx, int ny) {
    NscLayout L;
    L.tiles_x = (nx + nsc::TX - 1) / nsc::TX;
    L.tiles = int64_t(L.tiles_x) * ((ny + nsc::TY - 1) / nsc::TY);
    size_t o = kCtrlBytes;
    L.off_dt = o;
    o = align_up(o + size_t(L.tiles) * 4, 256);
    L.off_ws = o;
    o = align_up(o + size_t(L.tiles) * 4, 256);
    L.off_sq = o;
    o = align_up(o + size_t(L.tiles) * 32, 256);
    L.total = o;
    return L;
}

}  // namespace

extern "C" {

size_t cspb_ns_comp_workspace_bytes(int32_t nx, int32_t ny) {
    if (nx < 4 || ny < 4) return 0;
    return nsc_layout(nx, ny).total;
}

int cspb_ns_compressible(const cspb_ns_comp_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (d->nx < 4 || d->ny < 4 || !d->U || !d->R || !d->diag) return CSPB_ERR_ARGUMENT;
    if (int64_t(d->nx) * d->ny > (int64_t(1) << 31)) return CSPB_ERR_ARGUMENT;
    if (d->limiter != 0 && d->limiter != 1) return CSPB_ERR_UNSUPPORTED;
    if (d->walls != 0 && d->walls != 1) return CSPB_ERR_ARGUMENT;
    const NscLayout L = nsc_layout(d->nx, d->ny);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    if (L.tiles > 0x7fffffff) return CSPB_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(d->workspace);
    if (cudaMemsetAsync(ws, 0, kCtrlBytes, st) != cudaSuccess) return CSPB_ERR_CUDA;
    nsc::K g{};
    g.nx = d->nx;
    g.ny = d->ny;
    g.walls = d->walls;
    g.tiles_x = L.tiles_x;
    g.tiles = L.tiles;
    g.U = d->U;
    g.R = d->R;
    g.diag = d->diag;
    g.det_sq64 = d->det_sq64;
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    g.part_dt = reinterpret_cast<float*>(ws + L.off_dt);
    g.part_ws = reinterpret_cast<float*>(ws + L.off_ws);
    g.part_sq = reinterpret_cast<double*>(ws + L.off_sq);
    const size_t smem = sizeof(nsc::Smem);
    auto kern = d->limiter == 0 ? nsc::k_ns_comp<0> : nsc::k_ns_comp<1>;
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)) != cudaSuccess)
        return CSPB_ERR_CUDA;
    kern<<<unsigned(L.tiles), nsc::kThreads, smem, st>>>(g);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
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
