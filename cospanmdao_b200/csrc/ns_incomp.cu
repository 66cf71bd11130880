// ns_incomp.cu — the incompressible Navier-Stokes residual on a 2D periodic collocated grid, one streaming kernel.
//
//   r_u = u·∂u/∂x + v·∂u/∂y + ∂p/∂x − ν∇²u
//   r_v = u·∂v/∂x + v·∂v/∂y + ∂p/∂y − ν∇²v
//   r_c = ∂u/∂x + ∂v/∂y
// with ∂f/∂x ≈ (f[i+1] − f[i−1]) / 2h and ∇²f ≈ ((f[i+1]−f) + (f[i−1]−f) + (f[j+1]−f) + (f[j−1]−f)) / h². The
// neighbour differences are formed first: fields whose neighbours lie within a factor 2 of each other subtract exactly
// in f32 (Sterbenz), so the only roundings are the few that follow.
//
// No reference code computes this residual (the reference's ns-residual is the compressible one, ns_comp.cu); the
// formula is the workload's definition, and the oracle is an f64 restatement of it.
//
// Layout: u, v, p and r_u, r_v, r_c are (ny, nx) row-major. 16-byte aligned fields whose rows are whole 16-byte
// chunks (nx % 4 == 0 in f32, nx % 8 == 0 in bf16) take the block-tile path (nsi_tile below). Otherwise (unaligned or
// ragged rows) the register path:
// work item = one warp on a strip of 32·VEC columns × H rows:
// each lane owns 4 consecutive cells of a row (one 16-byte f32 / 8-byte bf16 load per field per row), x-neighbours come from the
// adjacent lanes by shuffle (the warp's edge lanes load one wrapped scalar), and the warp marches down its rows
// keeping the rows above and below in registers, two rows of loads in flight. Each input is read from HBM once (the
// 2 halo rows of a strip are L2 hits of the neighbouring strip); 24 B/cell in f32 storage, 18 B/cell in bf16.
//
// The three squared norms are accumulated per thread in f64, reduced per warp by a fixed xor tree, per block in warp
// order, and across blocks in block order by the last block to finish: bit-identical on every run.
#include "common.cuh"

namespace cspb {

constexpr int kNsiThreads = 256;
constexpr int kNsiWarps = kNsiThreads / 32;

struct NsiK {
    int nx, ny, H;
    int segs;          // column segments of 32·VEC cells
    int64_t items;     // segs × row strips
    float inv2h, invh2, nu;
    const void *u, *v, *p;
    float *ru, *rv, *rc;
    double* norms;
    double* part;      // [blocks][3]
    uint32_t* ctrl;
    // a y-slab of a larger grid (tile path only): the rows above and below the slab come from these rows of u, v, p
    // (nx floats each) instead of wrapping, and `norms` receives the squared sums, not their roots
    const float* up[3];
    const float* dn[3];
    int slab;
};

template <typename T, int VEC>
struct NsiRow {
    float c[VEC];  // this lane's cells
    float l, r;    // the wrapped neighbours outside the lane's cells when this lane needs them from memory
};

// ---- the residual of a cell, every rounding written out ------------------------------------------------------------
//   dfdx = (fE − fW)·inv2h, dfdy = (fN − fS)·inv2h, lap f = (((fE − fc) + (fW − fc)) + ((fN − fc) + (fS − fc)))·invh2
//   r_u = fma(−ν, lap u, fma(u, dudx, v·dudy) + dpdx), r_v = fma(−ν, lap v, fma(u, dvdx, v·dvdy) + dpdy),
//   r_c = dudx + dvdy
// Each operation is rounded to nearest on its own (the fused multiply-adds are the two written), so the compiler has
// no contraction left to choose. NsiOne evaluates one cell with the scalar instructions; NsiTwo two cells at once with
// Blackwell's packed f32x2 instructions (.rn, no flush to zero), which round each lane exactly as the scalar
// instruction would: both give the same bits for a cell, and the tile paths (pairs) and the register path (single
// cells) agree.
struct NsiOne {
    using V = float;
    static __device__ __forceinline__ V sp(float a) { return a; }
    static __device__ __forceinline__ V add(V a, V b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ V sub(V a, V b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ V mul(V a, V b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ V fma(V a, V b, V c) { return __fmaf_rn(a, b, c); }
};
struct NsiTwo {
    using V = float2;
    static __device__ __forceinline__ V sp(float a) { return make_float2(a, a); }
    static __device__ __forceinline__ V add(V a, V b) {
        V d;
        asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
            "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
            : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
        return d;
    }
    static __device__ __forceinline__ V sub(V a, V b) {
        V d;
        asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
            "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
            : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
        return d;
    }
    static __device__ __forceinline__ V mul(V a, V b) {
        V d;
        asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
            "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
            : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
        return d;
    }
    static __device__ __forceinline__ V fma(V a, V b, V c) {
        V d;
        asm("{\n\t.reg .b64 ra, rb, rc, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
            "mov.b64 rc, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rc;\n\tmov.b64 {%0, %1}, rd;\n\t}"
            : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
        return d;
    }
};
// The 5-point values of one field around a cell (or a pair of cells): centre, west, east, south, north.
template <class A>
struct NsiStar {
    typename A::V c, w, e, s, n;
};
template <class A>
__device__ __forceinline__ void nsi_cell(const NsiStar<A>& u, const NsiStar<A>& v, const NsiStar<A>& p, float inv2h,
                                         float invh2, float nu, typename A::V& ru, typename A::V& rv,
                                         typename A::V& rc) {
    using V = typename A::V;
    const V i2h = A::sp(inv2h), ih2 = A::sp(invh2), mnu = A::sp(-nu);
    const V dudx = A::mul(A::sub(u.e, u.w), i2h), dudy = A::mul(A::sub(u.n, u.s), i2h);
    const V dvdx = A::mul(A::sub(v.e, v.w), i2h), dvdy = A::mul(A::sub(v.n, v.s), i2h);
    const V dpdx = A::mul(A::sub(p.e, p.w), i2h), dpdy = A::mul(A::sub(p.n, p.s), i2h);
    const V lapu = A::mul(A::add(A::add(A::sub(u.e, u.c), A::sub(u.w, u.c)), A::add(A::sub(u.n, u.c), A::sub(u.s, u.c))),
                          ih2);
    const V lapv = A::mul(A::add(A::add(A::sub(v.e, v.c), A::sub(v.w, v.c)), A::add(A::sub(v.n, v.c), A::sub(v.s, v.c))),
                          ih2);
    ru = A::fma(mnu, lapu, A::add(A::fma(u.c, dudx, A::mul(v.c, dudy)), dpdx));
    rv = A::fma(mnu, lapv, A::add(A::fma(u.c, dvdx, A::mul(v.c, dvdy)), dpdy));
    rc = A::add(dudx, dvdy);
}

template <typename T>
__device__ __forceinline__ float ld1(const T* p, int64_t i) {
    if constexpr (sizeof(T) == 4) return __ldg(reinterpret_cast<const float*>(p) + i);
    else return __bfloat162float(p[i]);
}

template <typename T, int VEC>
__device__ __forceinline__ void load_cells(const T* f, int64_t rowoff, int c0, int ncols, float (&out)[VEC]) {
    if constexpr (VEC == 4 && sizeof(T) == 4) {
        if (ncols == 4) {
            const float4 q = ld_stream_f4(reinterpret_cast<const float*>(f) + rowoff + c0);
            out[0] = q.x; out[1] = q.y; out[2] = q.z; out[3] = q.w;
            return;
        }
    } else if constexpr (VEC == 4 && sizeof(T) == 2) {
        if (ncols == 4) {
            const uint2 q = ld_stream_u2(f + rowoff + c0);
            out[0] = bf16_lo(q.x); out[1] = bf16_hi(q.x); out[2] = bf16_lo(q.y); out[3] = bf16_hi(q.y);
            return;
        }
    }
#pragma unroll
    for (int e = 0; e < VEC; ++e) out[e] = e < ncols ? ld1(f, rowoff + c0 + e) : 0.f;
}

template <typename T, int VEC>
__device__ __forceinline__ void load_row(const T* f, int nx, int64_t rowoff, int c0, int ncols, bool need_l, bool need_r,
                                         NsiRow<T, VEC>& row) {
    load_cells<T, VEC>(f, rowoff, c0, ncols, row.c);
    row.l = need_l ? ld1(f, rowoff + (c0 == 0 ? nx - 1 : c0 - 1)) : 0.f;
    row.r = need_r ? ld1(f, rowoff + ((c0 + ncols) % nx)) : 0.f;
}

// x-neighbours of the lane's cells: left of cell 0 and right of cell VEC-1, from the adjacent lanes or memory.
template <typename T, int VEC>
__device__ __forceinline__ void x_neighbours(const NsiRow<T, VEC>& row, bool need_l, bool need_r, float& left, float& right) {
    const float from_left = __shfl_up_sync(0xffffffffu, row.c[VEC - 1], 1);
    const float from_right = __shfl_down_sync(0xffffffffu, row.c[0], 1);
    left = need_l ? row.l : from_left;
    right = need_r ? row.r : from_right;
}

// ---- block tiles (cp.async) -------------------------------------------------------------------------------------
// A block computes one tile of kNsiTileCols × kNsiTileRows cells. It first copies the tile's rows of u, v, p with the
// rows above and below it and the two wrapped halo columns into shared memory (cp.async: each warp takes every 8th
// row, its lanes the row's 16-byte chunks, then lane 0 and the last active lane the halo cells), waits once, then
// computes its rows from shared memory and stores the residuals. Four such tiles per SM are in flight while other
// tiles compute. The fields stay in their storage type in shared memory (bf16 is widened as it is read).
// Tile shapes (measured on B200 at 4096², the same per-cell bits whatever the shape): f32 128 × 32 (512-byte row runs;
// 256 × 16 and 512 × 8 ran alike); bf16 512 × 16, whose 1 KB row runs took 0.059 ms against 0.072 ms for 128 × 32
// (256-byte runs) with the same shared memory per tile. A tile row is [C0 - 1] the cell left of the tile,
// [C0 .. C0 + cols) its cells, [C0 + cols] the cell right, C0 = 16 B / sizeof(T).
template <typename T> inline constexpr int kNsiTileCols = sizeof(T) == 4 ? 128 : 512;
template <typename T> inline constexpr int kNsiTileRows = sizeof(T) == 4 ? 32 : 16;
template <typename T> inline constexpr int kNsiCell0 = 16 / int(sizeof(T));                             // 4 f32, 8 bf16
template <typename T> inline constexpr int kNsiPitch = kNsiCell0<T> + kNsiTileCols<T> + kNsiCell0<T>;  // 136, 528
template <typename T>  // 55,488 B (f32), 57,024 B (bf16)
inline constexpr size_t kNsiTileBytes = size_t(3) * (kNsiTileRows<T> + 2) * kNsiPitch<T> * sizeof(T);

template <typename T>
__host__ __device__ inline int64_t nsi_tiles(int nx, int ny) {
    return int64_t((nx + kNsiTileCols<T> - 1) / kNsiTileCols<T>) * ((ny + kNsiTileRows<T> - 1) / kNsiTileRows<T>);
}
__host__ __device__ inline int64_t nsi_tiles(bool bf16, int nx, int ny) {
    return bf16 ? nsi_tiles<__nv_bfloat16>(nx, ny) : nsi_tiles<float>(nx, ny);
}
// The tile path takes 16-byte aligned fields (checked by the caller) whose rows are whole 16-byte chunks: nx % 4 == 0
// in f32, nx % 8 == 0 in bf16. Single calls and task tables use this same rule, so a grid's decomposition (and hence
// its norms' bits) does not depend on how it was launched.
__host__ __device__ inline bool nsi_tile_rows(bool bf16, int nx) { return nx % (bf16 ? 8 : 4) == 0; }

__device__ __forceinline__ uint32_t nsi_smem(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void nsi_cp16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(nsi_smem(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void nsi_cp4(void* dst, const void* src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(nsi_smem(dst)), "l"(src) : "memory");
}
// 4 consecutive cells of a tile row in shared memory (16-byte aligned in f32, 8-byte in bf16), widened to f32
template <typename T>
__device__ __forceinline__ void nsi_ld4(const T* p, float (&c)[4]) {
    if constexpr (sizeof(T) == 4) {
        const float4 q = *reinterpret_cast<const float4*>(p);
        c[0] = q.x; c[1] = q.y; c[2] = q.z; c[3] = q.w;
    } else {
        const uint2 q = *reinterpret_cast<const uint2*>(p);
        c[0] = bf16_lo(q.x); c[1] = bf16_hi(q.x); c[2] = bf16_lo(q.y); c[3] = bf16_hi(q.y);
    }
}
template <typename T>
__device__ __forceinline__ float nsi_ld1(const T* p) {
    if constexpr (sizeof(T) == 4) return *p;
    else return __bfloat162float(*p);
}

template <typename T, int FIELD>
__device__ __forceinline__ void nsi_tile_compute(const NsiK& g, const T* buf, int x0, int y0, int scols, int th,
                                                 double& su, double& sv, double& sc);

// Tile b of a residual whose rows satisfy nsi_tile_rows. The residuals are the register path's (nsi_cell); each lane's
// 4 squares are summed in f32 (cells 0 and 2, cells 1 and 3, then the two sums) before one f64 addition per norm.
template <typename T>
__device__ __forceinline__ void nsi_tile(const NsiK& g, int64_t b, T* buf, double& su, double& sv, double& sc) {
    constexpr int C0 = kNsiCell0<T>, PITCH = kNsiPitch<T>, COLS = kNsiTileCols<T>, ROWS = kNsiTileRows<T>;
    constexpr int VC = 16 / int(sizeof(T));            // cells per 16-byte copy
    constexpr int kField = (ROWS + 2) * PITCH;         // elements between the fields
    const int tilesx = (g.nx + COLS - 1) / COLS;
    const int x0 = int(b % tilesx) * COLS, y0 = int(b / tilesx) * ROWS;
    const int scols = g.nx - x0 >= COLS ? COLS : g.nx - x0;  // a multiple of VC
    const int th = g.ny - y0 >= ROWS ? ROWS : g.ny - y0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lcol = x0 == 0 ? g.nx - 1 : x0 - 1;
    const int rcol = (x0 + scols) % g.nx;
    const int64_t nx = g.nx;
    const T* U = static_cast<const T*>(g.u);
    const T* V = static_cast<const T*>(g.v);
    const T* P = static_cast<const T*>(g.p);
    // tile row r holds grid row y0 - 1 + r (wrapped, or a slab's halo row), r = 0 .. th + 1
    auto row_src = [&](int r, const T*& ru_, const T*& rv_, const T*& rp_) {
        int gy = y0 - 1 + r;
        if constexpr (sizeof(T) == 4) {  // slabs are f32
            if (g.slab && gy < 0) {
                ru_ = g.up[0]; rv_ = g.up[1]; rp_ = g.up[2];
                return;
            }
            if (g.slab && gy >= g.ny) {
                ru_ = g.dn[0]; rv_ = g.dn[1]; rp_ = g.dn[2];
                return;
            }
        }
        gy = gy < 0 ? gy + g.ny : (gy >= g.ny ? gy - g.ny : gy);
        const int64_t ro = int64_t(gy) * nx;
        ru_ = U + ro; rv_ = V + ro; rp_ = P + ro;
    };
    // The halo cells, by 4-byte copies. In bf16 a copy moves the aligned pair of cells that holds the halo cell: the
    // left halo column is odd (x0 - 1 with x0 a multiple of 512, or nx - 1 with nx even), so its pair starts one cell
    // before it, at C0 - 2; the right one is even (a multiple of 8, or 0) and its pair starts at it, at C0 + scols (the
    // pair's second cell, inside the grid, lands in the pitch's padding).
    constexpr int kHaloL = sizeof(T) == 4 ? 0 : 1;  // cells the left copy starts before the halo cell
    const int last = (scols - 1) / VC % 32;         // the lane holding the row's last chunk
    for (int r = warp; r < th + 2; r += kNsiWarps) {
        const T *ru_, *rv_, *rp_;
        row_src(r, ru_, rv_, rp_);
        T* row = buf + r * PITCH;
#pragma unroll
        for (int k = 0; k < (COLS / VC + 31) / 32; ++k) {
            const int cc = (k * 32 + lane) * VC;  // this lane's chunks of the row
            if (cc < scols) {
                nsi_cp16(row + C0 + cc, ru_ + x0 + cc);
                nsi_cp16(row + kField + C0 + cc, rv_ + x0 + cc);
                nsi_cp16(row + 2 * kField + C0 + cc, rp_ + x0 + cc);
            }
        }
        if (lane == 0) {
            nsi_cp4(row + C0 - 1 - kHaloL, ru_ + lcol - kHaloL);
            nsi_cp4(row + kField + C0 - 1 - kHaloL, rv_ + lcol - kHaloL);
            nsi_cp4(row + 2 * kField + C0 - 1 - kHaloL, rp_ + lcol - kHaloL);
        }
        if (lane == last) {
            nsi_cp4(row + C0 + scols, ru_ + rcol);
            nsi_cp4(row + kField + C0 + scols, rv_ + rcol);
            nsi_cp4(row + 2 * kField + C0 + scols, rp_ + rcol);
        }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    __syncthreads();
    nsi_tile_compute<T, kField>(g, buf, x0, y0, scols, th, su, sv, sc);
}

// The residuals of one tile staged in shared memory (row r of field f at buf + f·FIELD + r·PITCH, cell x0 + c at
// column C0 + c, the halo cells at C0 - 1 and C0 + scols, tile row r = grid row y0 - 1 + r): the register path's
// arithmetic (nsi_cell, two cells per packed instruction); each lane's 4 squares are summed in f32 (cells 0 and 2,
// cells 1 and 3, then the two sums) before one f64 addition per norm. Warp w computes the items w, w + 8, ... of the
// tile (item = row × segments + segment).
template <typename T, int FIELD>
__device__ __forceinline__ void nsi_tile_compute(const NsiK& g, const T* buf, int x0, int y0, int scols, int th,
                                                 double& su, double& sv, double& sc) {
    constexpr int C0 = kNsiCell0<T>, PITCH = kNsiPitch<T>;
    constexpr int kField = FIELD;
    constexpr int SEGS = kNsiTileCols<T> / 128;  // segments of a tile row: 32 lanes × 4 cells each
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t nx = g.nx;
    const float inv2h = g.inv2h, invh2 = g.invh2, nu = g.nu;
    // item = tile row j × SEGS + segment; warp w takes items w, w + 8, ... (in f32 a tile row is one segment)
    for (int it = warp; it < th * SEGS; it += kNsiWarps) {
        const int j = it / SEGS, xs = (it % SEGS) * 128 + lane * 4;  // the lane's first cell within the tile
        if (xs >= scols) continue;                                     // past the tile's last cell
        const int c0 = x0 + xs;
        const T* const mine = buf + C0 + xs;
        const T* a = mine + (j + 1) * PITCH;
        const T* mS = mine + j * PITCH;
        const T* mN = mine + (j + 2) * PITCH;
        float cu[6], cv[6], cp[6];  // W, 4 cells, E of the row
        float uS[4], uN[4], vS[4], vN[4], pS[4], pN[4];
        {
            float ua[4], va[4], pa[4];
            nsi_ld4(a, ua);
            nsi_ld4(a + kField, va);
            nsi_ld4(a + 2 * kField, pa);
            cu[0] = nsi_ld1(a - 1); cu[5] = nsi_ld1(a + 4);
            cv[0] = nsi_ld1(a + kField - 1); cv[5] = nsi_ld1(a + kField + 4);
            cp[0] = nsi_ld1(a + 2 * kField - 1); cp[5] = nsi_ld1(a + 2 * kField + 4);
#pragma unroll
            for (int e = 0; e < 4; ++e) { cu[e + 1] = ua[e]; cv[e + 1] = va[e]; cp[e + 1] = pa[e]; }
            nsi_ld4(mS, uS);
            nsi_ld4(mN, uN);
            nsi_ld4(mS + kField, vS);
            nsi_ld4(mN + kField, vN);
            nsi_ld4(mS + 2 * kField, pS);
            nsi_ld4(mN + 2 * kField, pN);
        }
        // cells (0, 1) and (2, 3) as pairs
        float2 ru[2], rv[2], rc[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int e = 2 * h;
            const NsiStar<NsiTwo> su2{make_float2(cu[e + 1], cu[e + 2]), make_float2(cu[e], cu[e + 1]),
                                      make_float2(cu[e + 2], cu[e + 3]), make_float2(uS[e], uS[e + 1]),
                                      make_float2(uN[e], uN[e + 1])};
            const NsiStar<NsiTwo> sv2{make_float2(cv[e + 1], cv[e + 2]), make_float2(cv[e], cv[e + 1]),
                                      make_float2(cv[e + 2], cv[e + 3]), make_float2(vS[e], vS[e + 1]),
                                      make_float2(vN[e], vN[e + 1])};
            const NsiStar<NsiTwo> sp2{make_float2(cp[e + 1], cp[e + 2]), make_float2(cp[e], cp[e + 1]),
                                      make_float2(cp[e + 2], cp[e + 3]), make_float2(pS[e], pS[e + 1]),
                                      make_float2(pN[e], pN[e + 1])};
            nsi_cell<NsiTwo>(su2, sv2, sp2, inv2h, invh2, nu, ru[h], rv[h], rc[h]);
        }
        // squares: lane x of the pair sums cells 0 and 2, lane y cells 1 and 3, then x + y
        const float2 qu = NsiTwo::fma(ru[1], ru[1], NsiTwo::mul(ru[0], ru[0]));
        const float2 qv = NsiTwo::fma(rv[1], rv[1], NsiTwo::mul(rv[0], rv[0]));
        const float2 qc = NsiTwo::fma(rc[1], rc[1], NsiTwo::mul(rc[0], rc[0]));
        su += double(__fadd_rn(qu.x, qu.y));
        sv += double(__fadd_rn(qv.x, qv.y));
        sc += double(__fadd_rn(qc.x, qc.y));
        const int64_t ro = int64_t(y0 + j) * nx + c0;
        st_f4(g.ru + ro, make_float4(ru[0].x, ru[0].y, ru[1].x, ru[1].y));
        st_f4(g.rv + ro, make_float4(rv[0].x, rv[0].y, rv[1].x, rv[1].y));
        st_f4(g.rc + ro, make_float4(rc[0].x, rc[0].y, rc[1].x, rc[1].y));
    }
}

// The per-warp sums of nsi_partial and nsi_final, one array for both (they never overlap in time): four bf16 tiles
// per SM leave room for 200 bytes of static shared memory per block, not for two such arrays.
__device__ __forceinline__ double (*nsi_red())[3] {
    __shared__ double s_red[kNsiWarps][3];
    return s_red;
}

// The norm partial of block (or tile) b: a warp xor tree, the block in warp order, into part[b]. FENCE: make the
// partial visible and close with a barrier; without, the caller fences after its last partial, and the next s_part
// stores wait for the caller's next barrier.
template <bool FENCE = true>
__device__ __forceinline__ void nsi_partial(const NsiK& g, int64_t b, double su, double sv, double sc) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        su += __shfl_xor_sync(0xffffffffu, su, off);
        sv += __shfl_xor_sync(0xffffffffu, sv, off);
        sc += __shfl_xor_sync(0xffffffffu, sc, off);
    }
    double (*const s_part)[3] = nsi_red();
    if (lane == 0) { s_part[warp][0] = su; s_part[warp][1] = sv; s_part[warp][2] = sc; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = s_part[0][threadIdx.x];
        for (int w = 1; w < kNsiWarps; ++w) t += s_part[w][threadIdx.x];
        g.part[b * 3 + threadIdx.x] = t;
        if (FENCE) __threadfence();  // visible before any completion count taken after the barrier
    }
    if (FENCE) __syncthreads();
}

// The norms from the partials of blocks 0 .. nblocks-1, by the whole calling block in a fixed assignment and order
// (thread t < 256 the partials t, t + 256, ... in order, an xor tree per warp, warps 0..7 in order). Bit-identical on
// every run. Every thread of the block calls it (it holds a barrier); threads past 256 add nothing.
__device__ __forceinline__ void nsi_final(const NsiK& g, int64_t nblocks) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double (*const s_red)[3] = nsi_red();
    __threadfence();
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    const int64_t start = threadIdx.x < kNsiThreads ? int64_t(threadIdx.x) : nblocks;
    for (int64_t q = start; q < nblocks; q += kNsiThreads) {
        a0 += __ldcg(g.part + q * 3 + 0);
        a1 += __ldcg(g.part + q * 3 + 1);
        a2 += __ldcg(g.part + q * 3 + 2);
    }
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, off);
        a1 += __shfl_xor_sync(0xffffffffu, a1, off);
        a2 += __shfl_xor_sync(0xffffffffu, a2, off);
    }
    if (lane == 0 && warp < kNsiWarps) { s_red[warp][0] = a0; s_red[warp][1] = a1; s_red[warp][2] = a2; }
    __syncthreads();
    if (threadIdx.x < 3 && g.norms) {
        double t = s_red[0][threadIdx.x];
        for (int w = 1; w < kNsiWarps; ++w) t += s_red[w][threadIdx.x];
        g.norms[threadIdx.x] = g.slab ? t : sqrt(t);  // a slab's squared sums are added across slabs first
    }
}

// The norms of block b: its partial into part[b]; the last block to finish (counter `done`) sums the partials.
__device__ __forceinline__ void nsi_norms(const NsiK& g, int64_t b, int64_t nblocks, uint32_t* done, double su,
                                          double sv, double sc) {
    __shared__ int s_last;
    nsi_partial(g, b, su, sv, sc);
    if (threadIdx.x == 0) {
        pdl_wait();  // the count lives in the control block a single call clears with a kernel ahead of this one
        s_last = atomicAdd(done, 1u) == uint32_t(nblocks - 1);
    }
    __syncthreads();
    if (s_last) nsi_final(g, nblocks);  // block-uniform
    __syncthreads();  // the shared memory of this block is reused by the next block of a persistent caller
}

// Tile b (of nblocks) of a residual, with its norms.
template <typename T>
__device__ __forceinline__ void nsi_tile_block(const NsiK& g, int64_t b, int64_t nblocks, uint32_t* done, T* buf) {
    double su = 0.0, sv = 0.0, sc = 0.0;
    nsi_tile<T>(g, b, buf, su, sv, sc);
    nsi_norms(g, b, nblocks, done, su, sv, sc);
}

// Block b (of nblocks) of one residual: its 8 warps take items 8b .. 8b+7. Its norm partial goes to part[b]; the last
// block to finish (counter `done`) sums the partials in block order.
template <typename T, int VEC>
__device__ __forceinline__ void nsi_block(const NsiK& g, int64_t b, int64_t nblocks, uint32_t* done) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t item = b * kNsiWarps + warp;
    double su = 0.0, sv = 0.0, sc = 0.0;
    if (item < g.items) {  // warp-uniform
        const int seg = int(item % g.segs);
        const int strip = int(item / g.segs);
        const int c0 = seg * 32 * VEC + lane * VEC;
        const int ncols = c0 >= g.nx ? 0 : (g.nx - c0 >= VEC ? VEC : g.nx - c0);
        const bool active = ncols > 0;
        // the lane needs its left neighbour from memory when it is the first lane; its right one when it is the
        // last lane of the warp or the last lane holding cells
        const bool need_l = lane == 0;
        const bool need_r = active && (lane == 31 || c0 + VEC >= g.nx);
        const int j0 = strip * g.H;
        const int j1 = min(g.ny, j0 + g.H);
        const T* U = static_cast<const T*>(g.u);
        const T* V = static_cast<const T*>(g.v);
        const T* P = static_cast<const T*>(g.p);
        const int64_t nx = g.nx;
        auto wrapj = [&](int j) { return j < 0 ? j + g.ny : (j >= g.ny ? j - g.ny : j); };

        NsiRow<T, VEC> u0, u1, u2, v0, v1, v2, p0, p1, p2;  // rows j-1, j, j+1
        NsiRow<T, VEC> u3, v3, p3;                          // row j+2 (in flight)
        {
            const int64_t ra = int64_t(wrapj(j0 - 1)) * nx, rb = int64_t(j0) * nx, rc = int64_t(wrapj(j0 + 1)) * nx;
            load_row<T, VEC>(U, g.nx, ra, c0, ncols, need_l, need_r, u0);
            load_row<T, VEC>(V, g.nx, ra, c0, ncols, need_l, need_r, v0);
            load_row<T, VEC>(P, g.nx, ra, c0, ncols, need_l, need_r, p0);
            load_row<T, VEC>(U, g.nx, rb, c0, ncols, need_l, need_r, u1);
            load_row<T, VEC>(V, g.nx, rb, c0, ncols, need_l, need_r, v1);
            load_row<T, VEC>(P, g.nx, rb, c0, ncols, need_l, need_r, p1);
            load_row<T, VEC>(U, g.nx, rc, c0, ncols, need_l, need_r, u2);
            load_row<T, VEC>(V, g.nx, rc, c0, ncols, need_l, need_r, v2);
            load_row<T, VEC>(P, g.nx, rc, c0, ncols, need_l, need_r, p2);
        }
        const float inv2h = g.inv2h, invh2 = g.invh2, nu = g.nu;
        for (int j = j0; j < j1; ++j) {
            if (j + 1 < j1) {  // prefetch row j+2 while row j is computed
                const int64_t rd = int64_t(wrapj(j + 2)) * nx;
                load_row<T, VEC>(U, g.nx, rd, c0, ncols, need_l, need_r, u3);
                load_row<T, VEC>(V, g.nx, rd, c0, ncols, need_l, need_r, v3);
                load_row<T, VEC>(P, g.nx, rd, c0, ncols, need_l, need_r, p3);
            }
            float ul, ur, vl, vr, pl, pr;
            x_neighbours<T, VEC>(u1, need_l, need_r, ul, ur);
            x_neighbours<T, VEC>(v1, need_l, need_r, vl, vr);
            x_neighbours<T, VEC>(p1, need_l, need_r, pl, pr);
            float oru[VEC], orv[VEC], orc[VEC];
#pragma unroll
            for (int e = 0; e < VEC; ++e) {
                const float uc = u1.c[e], vc = v1.c[e];
                const float uW = e == 0 ? ul : u1.c[e - 1], uE = e == VEC - 1 ? ur : u1.c[e + 1];
                const float vW = e == 0 ? vl : v1.c[e - 1], vE = e == VEC - 1 ? vr : v1.c[e + 1];
                const float pW = e == 0 ? pl : p1.c[e - 1], pE = e == VEC - 1 ? pr : p1.c[e + 1];
                const NsiStar<NsiOne> su1{uc, uW, uE, u0.c[e], u2.c[e]};
                const NsiStar<NsiOne> sv1{vc, vW, vE, v0.c[e], v2.c[e]};
                const NsiStar<NsiOne> sp1{p1.c[e], pW, pE, p0.c[e], p2.c[e]};
                float ru, rv, rc;
                nsi_cell<NsiOne>(su1, sv1, sp1, inv2h, invh2, nu, ru, rv, rc);
                oru[e] = ru; orv[e] = rv; orc[e] = rc;
                if (e < ncols) {
                    su = __fma_rn(double(ru), double(ru), su);
                    sv = __fma_rn(double(rv), double(rv), sv);
                    sc = __fma_rn(double(rc), double(rc), sc);
                }
            }
            const int64_t ro = int64_t(j) * nx + c0;
            if (ncols == VEC && (VEC % 4) == 0) {
#pragma unroll
                for (int q = 0; q < VEC / 4; ++q) {
                    st_f4(g.ru + ro + 4 * q, make_float4(oru[4 * q], oru[4 * q + 1], oru[4 * q + 2], oru[4 * q + 3]));
                    st_f4(g.rv + ro + 4 * q, make_float4(orv[4 * q], orv[4 * q + 1], orv[4 * q + 2], orv[4 * q + 3]));
                    st_f4(g.rc + ro + 4 * q, make_float4(orc[4 * q], orc[4 * q + 1], orc[4 * q + 2], orc[4 * q + 3]));
                }
            } else {
#pragma unroll
                for (int e = 0; e < VEC; ++e)
                    if (e < ncols) { g.ru[ro + e] = oru[e]; g.rv[ro + e] = orv[e]; g.rc[ro + e] = orc[e]; }
            }
            u0 = u1; u1 = u2; u2 = u3;
            v0 = v1; v1 = v2; v2 = v3;
            p0 = p1; p1 = p2; p2 = p3;
        }
    }
    nsi_norms(g, b, nblocks, done, su, sv, sc);
}

template <typename T, int VEC>
__global__ void __launch_bounds__(kNsiThreads) k_ns_incomp(NsiK g) {
    nsi_block<T, VEC>(g, blockIdx.x, gridDim.x, g.ctrl + kDone0);
}
// The tile path of one residual: launched with a block per tile, 4 blocks per SM (64 registers a thread at most).
// Measured on B200 at 4096²: a persistent grid (4 blocks per SM taking tiles k, k + grid, ...) ran 0.0914 / 0.0663 ms
// (f32 / bf16) against 0.0811 / 0.0616 ms for a block per tile, which the hardware hands out in tile order as blocks
// finish. The two storage types end a block in the form that measured faster for each (the same sums either way):
// f32 tiles as the task kernel's (0.0803 against 0.0810 ms), bf16 with one fence after the partial and no closing
// barrier (0.0617 against 0.0638 ms); the bf16 form takes any grid, a block's tiles in order.
template <typename T>
__global__ void __launch_bounds__(kNsiThreads, 4) k_ns_incomp_tile(NsiK g) {
    extern __shared__ __align__(16) unsigned char nsi_raw[];
    T* const buf = reinterpret_cast<T*>(nsi_raw);
    if constexpr (sizeof(T) == 4) {
        nsi_tile_block<T>(g, blockIdx.x, gridDim.x, g.ctrl + kDone0, buf);
    } else {
        __shared__ int s_last;
        const int64_t tiles = nsi_tiles<T>(g.nx, g.ny);
        for (int64_t b = blockIdx.x; b < tiles; b += gridDim.x) {
            double su = 0.0, sv = 0.0, sc = 0.0;
            nsi_tile<T>(g, b, buf, su, sv, sc);
            nsi_partial<false>(g, b, su, sv, sc);
        }
        if (threadIdx.x < 3) __threadfence();  // the partials this thread stored, before the count
        __syncthreads();
        if (threadIdx.x == 0) {
            pdl_wait();
            s_last = atomicAdd(g.ctrl + kDone0, 1u) == uint32_t(gridDim.x - 1);
        }
        __syncthreads();
        if (s_last) nsi_final(g, tiles);  // block-uniform
    }
}

// ---- many residuals in one persistent launch -----------------------------------------------------------------
// The row-strip height H of a grid: the one whose block count best fills whole waves of kNsiWave blocks (4 per SM on
// the 148 SMs of a B200; a constant, so that the decomposition and hence every sum depends on (nx, ny) alone), the
// taller one on a tie. Small grids take the shortest strips (the most blocks).
constexpr int64_t kNsiWave = 4 * 148;
__host__ __device__ inline void nsi_shape(int nx, int ny, int vec, int& H, int& segs, int64_t& items, int64_t& blocks) {
    segs = (nx + 32 * vec - 1) / (32 * vec);
    int64_t best_b = 0, best_w = 1;
    H = 32;
    for (int h = 32; h >= 4; h -= 4) {
        const int64_t b = (int64_t(segs) * ((ny + h - 1) / h) + kNsiWarps - 1) / kNsiWarps;
        const int64_t w = (b + kNsiWave - 1) / kNsiWave;
        if (b * best_w > best_b * w) {  // a higher fill b / (w · wave)
            best_b = b;
            best_w = w;
            H = h;
        }
    }
    items = int64_t(segs) * ((ny + H - 1) / H);
    blocks = (items + kNsiWarps - 1) / kNsiWarps;
}

__device__ __forceinline__ bool nsi_fast(const cspb_ns_incomp_task& t, int vfast) {
    auto al = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; };
    return al(t.u) && al(t.v) && al(t.p) && al(t.ru) && al(t.rv) && al(t.rc) && t.nx % vfast == 0;
}

struct NsiTasksK {
    const cspb_ns_incomp_task* tasks;
    int64_t count;
    int bf16;
    uint64_t* blocks;   // [count]
    uint64_t* boff;     // [count + 1]
    uint32_t* done;     // [count]
    double* part;       // [Σ blocks][3]
    uint64_t cap_blocks;
    uint32_t* ctrl;
};

__global__ void k_nsi_plan(NsiTasksK g) {
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < g.count; k += int64_t(gridDim.x) * blockDim.x) {
        const cspb_ns_incomp_task& t = g.tasks[k];
        uint64_t nb = 0;
        if (t.nx >= 3 && t.ny >= 3 && t.u && t.v && t.p && t.ru && t.rv && t.rc) {
            const bool fast = nsi_fast(t, 4);
            int H, segs;
            int64_t items, blocks;
            if (fast && nsi_tile_rows(g.bf16 != 0, t.nx)) blocks = nsi_tiles(g.bf16 != 0, t.nx, t.ny);  // tiles
            else nsi_shape(t.nx, t.ny, fast ? 4 : 1, H, segs, items, blocks);
            nb = uint64_t(blocks);
        } else {
            set_status(g.ctrl, CSPB_DEV_NEGATIVE);
        }
        g.blocks[k] = nb;
    }
}

// MINB: blocks per SM the registers must allow (4, so that tiles run 4 blocks per SM as in the single call)
template <typename T, int MINB>
__global__ void __launch_bounds__(kNsiThreads, MINB) k_nsi_tasks(NsiTasksK g) {
    extern __shared__ __align__(16) unsigned char nsi_raw[];
    __shared__ int s_go;
    if (threadIdx.x == 0) s_go = __ldcg(g.boff + g.count) <= g.cap_blocks && !status_bad(g.ctrl);
    __syncthreads();
    if (!s_go) {
        if (threadIdx.x == 0 && __ldcg(g.boff + g.count) > g.cap_blocks) set_status(g.ctrl, CSPB_DEV_CAPACITY);
        return;
    }
    const uint64_t total = __ldcg(g.boff + g.count);
    constexpr int vfast = 4;
    int64_t hint = 0;
    for (uint32_t v = grab_work(g.ctrl, kWork0); uint64_t(v) < total;) {
        const uint32_t next = prefetch_work(g.ctrl, kWork0);
        // the task of block v: boff[lo] <= v < boff[lo + 1]; a block's items increase, so start from its last task
        int64_t lo = 0, hi = g.count;
        const uint64_t ha = __ldcg(g.boff + hint), hb = __ldcg(g.boff + hint + 1);
        if (ha <= v && v < hb) {
            lo = hint;
            hi = hint + 1;
        } else if (ha <= v) {
            lo = hint;
            for (int64_t step = 1;; step <<= 1) {
                const int64_t t = lo + step;
                if (t >= g.count) break;
                if (__ldcg(g.boff + t) > v) { hi = t; break; }
                lo = t;
            }
        }
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (__ldcg(g.boff + mid) <= v) lo = mid; else hi = mid;
        }
        hint = lo;
        const cspb_ns_incomp_task& t = g.tasks[lo];
        const bool fast = nsi_fast(t, vfast);
        NsiK k{};
        int64_t blocks;
        const bool tile = fast && nsi_tile_rows(sizeof(T) == 2, t.nx);
        if (tile) blocks = nsi_tiles<T>(t.nx, t.ny);
        else nsi_shape(t.nx, t.ny, fast ? vfast : 1, k.H, k.segs, k.items, blocks);
        k.nx = t.nx;
        k.ny = t.ny;
        k.inv2h = float(1.0 / (2.0 * t.h));
        k.invh2 = float(1.0 / (t.h * t.h));
        k.nu = float(t.nu);
        k.u = t.u; k.v = t.v; k.p = t.p;
        k.ru = t.ru; k.rv = t.rv; k.rc = t.rc;
        k.norms = t.norms;
        k.part = g.part + 3 * __ldcg(g.boff + lo);
        k.ctrl = g.ctrl;
        const int64_t b = int64_t(v) - int64_t(__ldcg(g.boff + lo));
        if (tile) {
            nsi_tile_block<T>(k, b, blocks, g.done + lo, reinterpret_cast<T*>(nsi_raw));
        } else if constexpr (sizeof(T) == 2) {  // f32 fast tasks are tiles
            if (fast) nsi_block<T, vfast>(k, b, blocks, g.done + lo);
            else nsi_block<T, 1>(k, b, blocks, g.done + lo);
        } else {
            nsi_block<T, 1>(k, b, blocks, g.done + lo);
        }
        v = share_work(next);
    }
}

}  // namespace cspb

using namespace cspb;
using cspb_host::align_up;
using cspb_host::aligned;

namespace {

// An f32 tile needs more than the default 48 KB of dynamic shared memory per block.
bool tile_ready(const void* kern, size_t bytes) {
    return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)) == cudaSuccess;
}

struct NsiPlan {
    int vec = 4, H = 32, segs = 0;
    int64_t items = 0, blocks = 0;
    size_t ws = 0;
};

// The row-strip height depends on the grid alone (never on the device), so the sums run in the same order anywhere.
NsiPlan nsi_plan(int nx, int ny, int vec) {
    NsiPlan p;
    p.vec = vec;
    nsi_shape(nx, ny, vec, p.H, p.segs, p.items, p.blocks);
    p.ws = align_up(kCtrlBytes + size_t(p.blocks) * 3 * sizeof(double), 256);
    return p;
}

// The tile kernel over the tiles of one residual (or slab), a block per tile, after the kernel that clears the
// workspace's control block: it may start before that kernel ends and waits for it only at its completion count.
template <typename T>
int launch_tiles(NsiK g, cudaStream_t st) {
    const void* kern = reinterpret_cast<const void*>(k_ns_incomp_tile<T>);
    const int64_t tiles = nsi_tiles<T>(g.nx, g.ny);
    if (tiles > int64_t(0x7fffffff)) return CSPB_ERR_TOO_LARGE;  // the grid's x extent
    if (!tile_ready(kern, kNsiTileBytes<T>)) return CSPB_ERR_LAUNCH;
    const int rc = cspb_host::clear_ctrl(g.ctrl, st);
    if (rc != CSPB_OK) return rc;
    void* args[] = {&g};
    return cspb_host::launch_dependent(kern, dim3(unsigned(tiles)), dim3(kNsiThreads), kNsiTileBytes<T>, st, args);
}

struct NsiTasksLayout {
    size_t off_blocks = 0, off_boff = 0, off_done = 0, off_scan = 0, off_part = 0, total = 0;
    uint64_t cap_blocks = 0;
};

// Σ blocks over tasks <= max_cells/80 + 3·count. A task's blocks: register strips <= cells/1024 + (nx + ny)/32 + 2;
// f32 tiles <= cells/4096 + nx/128 + ny/32 + 1; bf16 tiles <= cells/8192 + nx/512 + ny/16 + 1. Each is at most
// cells/80 + 3 for nx, ny >= 3 (the tiles take nx >= 4, nx >= 8 in bf16).
NsiTasksLayout nsi_tasks_layout(int64_t count, int64_t max_cells) {
    NsiTasksLayout L;
    L.cap_blocks = uint64_t(max_cells) / 80 + 3 * uint64_t(count);
    size_t o = kCtrlBytes;
    L.off_blocks = o;
    o = align_up(o + size_t(count) * 8, 256);
    L.off_boff = o;
    o = align_up(o + size_t(count + 1) * 8, 256);
    L.off_done = o;
    o = align_up(o + size_t(count) * 4, 256);
    L.off_scan = o;
    o = align_up(o + cspb_scan_workspace_bytes(count), 256);
    L.off_part = o;
    o = align_up(o + size_t(L.cap_blocks) * 3 * sizeof(double), 256);
    L.total = o;
    return L;
}

}  // namespace

extern "C" {

size_t cspb_ns_incomp_workspace_bytes(int32_t nx, int32_t ny) {
    if (nx < 3 || ny < 3) return 0;
    // the scalar plan (vec 1) or the tiles of either storage type: whichever has the most partials
    const int64_t nt = nsi_tiles<float>(nx, ny) > nsi_tiles<__nv_bfloat16>(nx, ny) ? nsi_tiles<float>(nx, ny)
                                                                                  : nsi_tiles<__nv_bfloat16>(nx, ny);
    const size_t tiles = align_up(kCtrlBytes + size_t(nt) * 3 * sizeof(double), 256);
    const size_t scalar = nsi_plan(nx, ny, 1).ws;
    return tiles > scalar ? tiles : scalar;
}

int cspb_ns_incompressible(const cspb_ns_incomp_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (d->nx < 3 || d->ny < 3) return CSPB_ERR_ARGUMENT;
    if (!d->u || !d->v || !d->p || !d->ru || !d->rv || !d->rc) return CSPB_ERR_ARGUMENT;
    if (!(d->h > 0.0) || !(d->nu >= 0.0)) return CSPB_ERR_ARGUMENT;
    if (d->dtype != CSPB_F32 && d->dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    if (d->flags != 0) return CSPB_ERR_UNSUPPORTED;
    const bool bf16 = d->dtype == CSPB_BF16;
    const int vfast = 4;  // 4 cells per lane: 16-byte loads in f32, 8-byte loads in bf16
    const bool in_al = aligned(d->u, 16) && aligned(d->v, 16) && aligned(d->p, 16);
    const bool out_al = aligned(d->ru, 16) && aligned(d->rv, 16) && aligned(d->rc, 16);
    const bool fast = in_al && out_al && d->nx % vfast == 0;
    NsiPlan P = nsi_plan(d->nx, d->ny, fast ? vfast : 1);
    const bool tile = fast && nsi_tile_rows(bf16, d->nx);
    if (tile) {
        P.blocks = nsi_tiles(bf16, d->nx, d->ny);
        P.ws = align_up(kCtrlBytes + size_t(P.blocks) * 3 * sizeof(double), 256);
    }
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < P.ws) return CSPB_ERR_WORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the tiles clear the control block themselves (launch_tiles); the register path after a memset
    if (!tile && cudaMemsetAsync(d->workspace, 0, kCtrlBytes, st) != cudaSuccess) return CSPB_ERR_CUDA;
    NsiK g{};
    g.nx = d->nx;
    g.ny = d->ny;
    g.H = P.H;
    g.segs = P.segs;
    g.items = P.items;
    g.inv2h = float(1.0 / (2.0 * d->h));
    g.invh2 = float(1.0 / (d->h * d->h));
    g.nu = float(d->nu);
    g.u = d->u; g.v = d->v; g.p = d->p;
    g.ru = d->ru; g.rv = d->rv; g.rc = d->rc;
    g.norms = d->norms;
    g.ctrl = static_cast<uint32_t*>(d->workspace);
    g.part = reinterpret_cast<double*>(static_cast<char*>(d->workspace) + kCtrlBytes);
    // aligned fields with whole 16-byte rows: the tiles; otherwise the register path, a block per item
    if (tile) return bf16 ? launch_tiles<__nv_bfloat16>(g, st) : launch_tiles<float>(g, st);
    const dim3 grid(unsigned(P.blocks)), block(kNsiThreads);
    if (bf16) {
        if (fast) k_ns_incomp<__nv_bfloat16, 4><<<grid, block, 0, st>>>(g);
        else k_ns_incomp<__nv_bfloat16, 1><<<grid, block, 0, st>>>(g);
    } else {
        k_ns_incomp<float, 1><<<grid, block, 0, st>>>(g);
    }
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

size_t cspb_ns_incomp_tasks_workspace_bytes(int64_t count, int64_t max_cells) {
    if (count < 1 || max_cells < 1) return 0;
    return nsi_tasks_layout(count, max_cells).total;
}

int cspb_ns_incomp_tasks(const cspb_ns_incomp_task* tasks, int64_t count, int64_t max_cells, int32_t dtype,
                         void* workspace, size_t workspace_bytes, void* stream) {
    if (!tasks || count < 1 || count > (int64_t(1) << 26) || max_cells < 1) return CSPB_ERR_ARGUMENT;
    if (dtype != CSPB_F32 && dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    const NsiTasksLayout L = nsi_tasks_layout(count, max_cells);
    if (!workspace || !aligned(workspace, 256) || workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    if (L.cap_blocks >= 0xffffffffull) return CSPB_ERR_ARGUMENT;
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(workspace);
    if (cudaMemsetAsync(ws, 0, kCtrlBytes, st) != cudaSuccess) return CSPB_ERR_CUDA;
    if (cudaMemsetAsync(ws + L.off_done, 0, size_t(count) * 4, st) != cudaSuccess) return CSPB_ERR_CUDA;
    NsiTasksK g{};
    g.tasks = tasks;
    g.count = count;
    g.bf16 = dtype == CSPB_BF16;
    g.blocks = reinterpret_cast<uint64_t*>(ws + L.off_blocks);
    g.boff = reinterpret_cast<uint64_t*>(ws + L.off_boff);
    g.done = reinterpret_cast<uint32_t*>(ws + L.off_done);
    g.part = reinterpret_cast<double*>(ws + L.off_part);
    g.cap_blocks = L.cap_blocks;
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    int64_t pb = (count + 255) / 256;
    if (pb > 4096) pb = 4096;
    k_nsi_plan<<<unsigned(pb), 256, 0, st>>>(g);
    if (cudaGetLastError() != cudaSuccess) return CSPB_ERR_LAUNCH;
    const int r = cspb_exclusive_scan_u64(g.blocks, g.boff, count, ws + L.off_scan, cspb_scan_workspace_bytes(count),
                                          stream);
    if (r != CSPB_OK) return r;
    const void* kern = g.bf16 ? reinterpret_cast<const void*>(k_nsi_tasks<__nv_bfloat16, 4>)
                              : reinterpret_cast<const void*>(k_nsi_tasks<float, 4>);
    const size_t smem = g.bf16 ? kNsiTileBytes<__nv_bfloat16> : kNsiTileBytes<float>;
    if (!tile_ready(kern, smem)) return CSPB_ERR_LAUNCH;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kNsiThreads, smem) != cudaSuccess || per_sm < 1)
        return CSPB_ERR_LAUNCH;
    void* args[] = {&g};
    if (cudaLaunchKernel(kern, dim3(unsigned(per_sm * di.sms)), dim3(kNsiThreads), args, smem, st) != cudaSuccess)
        return CSPB_ERR_LAUNCH;
    return CSPB_OK;
}

size_t cspb_ns_incomp_slab_workspace_bytes(int32_t nx, int32_t rows) {
    if (nx < 3 || rows < 1) return 0;
    return align_up(kCtrlBytes + size_t(nsi_tiles<float>(nx, rows)) * 3 * sizeof(double), 256);
}

int cspb_ns_incomp_slab(const cspb_ns_incomp_slab_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (d->nx < 3 || d->rows < 1) return CSPB_ERR_ARGUMENT;
    if (!d->u || !d->v || !d->p || !d->ru || !d->rv || !d->rc || !d->sums) return CSPB_ERR_ARGUMENT;
    for (int f = 0; f < 3; ++f)
        if (!d->up[f] || !d->dn[f]) return CSPB_ERR_ARGUMENT;
    if (!(d->h > 0.0) || !(d->nu >= 0.0)) return CSPB_ERR_ARGUMENT;
    if (d->flags != 0) return CSPB_ERR_UNSUPPORTED;
    // the tile path only: 16-byte aligned f32 rows
    bool al = d->nx % 4 == 0 && aligned(d->u, 16) && aligned(d->v, 16) && aligned(d->p, 16) && aligned(d->ru, 16) &&
              aligned(d->rv, 16) && aligned(d->rc, 16);
    for (int f = 0; f < 3; ++f) al = al && aligned(d->up[f], 16) && aligned(d->dn[f], 16);
    if (!al) return CSPB_ERR_UNSUPPORTED;
    const size_t need = cspb_ns_incomp_slab_workspace_bytes(d->nx, d->rows);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < need) return CSPB_ERR_WORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NsiK g{};  // launch_tiles clears the control block
    g.nx = d->nx;
    g.ny = d->rows;
    g.inv2h = float(1.0 / (2.0 * d->h));
    g.invh2 = float(1.0 / (d->h * d->h));
    g.nu = float(d->nu);
    g.u = d->u; g.v = d->v; g.p = d->p;
    g.ru = d->ru; g.rv = d->rv; g.rc = d->rc;
    g.norms = d->sums;
    g.ctrl = static_cast<uint32_t*>(d->workspace);
    g.part = reinterpret_cast<double*>(static_cast<char*>(d->workspace) + kCtrlBytes);
    for (int f = 0; f < 3; ++f) {
        g.up[f] = d->up[f];
        g.dn[f] = d->dn[f];
    }
    g.slab = 1;
    return launch_tiles<float>(g, st);
}

}  // extern "C"
