/*
 * cspb.h — the C ABI of libcspb.so, the B200 (sm_100a) kernels behind CoSpan's fused component chains.
 *
 * Every entry point is asynchronous on the given CUDA stream (passed as void*; NULL is the legacy default stream),
 * takes caller-owned device buffers and a caller-owned workspace, and never allocates. A call returns a host status
 * (CSPB_OK or a CSPB_ERR_* code) for what can be checked before the launch; what only the device can see (a bounded
 * wait that gave up, a ragged count that is negative or too large) is written to the status word at the start of the
 * workspace and read back by cspb_read_status() after the work has run. The one exception is
 * cspb_build_column_static, which takes no workspace: its scratch is a fixed array inside the library, and every
 * device-side condition it can meet (a negative count, a total past 2^32 - 1, a bounded wait that gave up) is reported
 * in the flag word it writes beside the total (CSPB_COLUMN_* bits below).
 *
 * The reference (NAGAGroup/CospanMDAO) has no C ABI: its kernels are SYCL bodies that AdaptiveCpp JIT-compiles and
 * launches from GroupLauncher::launch (cospanmdao/include/naga/cospan/component.hpp:779-970) through launch_group
 * (cospanmdao/include/naga/cospan/kernel.hpp:1015-1067). Each entry point below names the reference code whose
 * results it reproduces; a host runtime calls it where the reference submits the corresponding fused group.
 *
 * Thread safety: calls on distinct (stream, workspace) pairs may run concurrently. Two calls that share a workspace
 * must be ordered on one stream.
 */
#ifndef CSPB_H
#define CSPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------------------------------- */
enum {
    CSPB_OK = 0,
    CSPB_ERR_ARGUMENT = 1,    /* a size, pointer, stride or alignment the entry point rejects */
    CSPB_ERR_WORKSPACE = 2,   /* workspace NULL, misaligned or smaller than cspb_*_workspace_bytes() */
    CSPB_ERR_LAUNCH = 3,      /* a kernel launch failed (cudaGetLastError after the launch) */
    CSPB_ERR_TIMEOUT = 4,     /* device status: a bounded device-side wait gave up; outputs are not valid */
    CSPB_ERR_NEGATIVE = 5,    /* device status: a ragged count is negative, or offsets decrease or do not start at 0 */
    CSPB_ERR_EXCEEDS32 = 6,   /* device status: a ragged value or total is past 2^32 - 1 */
    CSPB_ERR_UNSUPPORTED = 7, /* a dtype / option combination this build does not provide */
    CSPB_ERR_CUDA = 8,        /* another CUDA runtime error (cudaMemsetAsync, cudaMemcpyAsync, ...) */
    CSPB_ERR_CAPACITY = 9,    /* device status: device-computed totals do not fit the capacities the caller declared */
    CSPB_ERR_TOO_LARGE = 10   /* the input is larger than the call allows (the fixed scratch of
                                 cspb_build_column_static; an NS grid of more than 2^31 - 1 tiles) */
};

/* bits of the device status word (the first 4 bytes of every workspace) */
#define CSPB_DEV_TIMEOUT 1u
#define CSPB_DEV_NEGATIVE 2u
#define CSPB_DEV_EXCEEDS32 4u
#define CSPB_DEV_CAPACITY 8u
#define CSPB_DEV_ARGUMENT 16u  /* a task contradicts a flag of the call (CSPB_BATCH_NO_B); read as CSPB_ERR_ARGUMENT */

/* bits of the flag word a ragged-column build writes to total_flag[1] (cspb_build_column, cspb_build_column_static).
 * 1 and 2 are the reference's own flags (cospanmdao/include/naga/cospan/shape_hook.hpp:455-463); 4 is this library's:
 * the device scan's bounded look-back gave up, so the offsets and the total are not valid. */
#define CSPB_COLUMN_NEGATIVE 1u
#define CSPB_COLUMN_EXCEEDS32 2u
#define CSPB_COLUMN_TIMEOUT 4u

/* storage dtypes of the big operands (the matrix of a GEMVER, the fields of a stencil) */
enum { CSPB_F32 = 0, CSPB_BF16 = 1 };

/* integer dtypes of a ragged count source (build_column) */
enum { CSPB_I32 = 0, CSPB_U32 = 1, CSPB_I64 = 2, CSPB_U64 = 3 };

/* A human-readable name of a status code. */
const char* cspb_status_string(int status);

/* The library's version string and the sm architecture it was built for (e.g. "cspb 0.1 sm_100a"). */
const char* cspb_version(void);

/* Synchronizes `stream`, reads the device status word of `workspace` and returns the CSPB_ERR_* code it holds
 * (CSPB_OK when clear). The raw word goes to *raw when raw is not NULL. */
int cspb_read_status(const void* workspace, uint32_t* raw, void* stream);

/* ==================================================================================================================
 * GEMVER:  Â = A + u1·v1ᵀ + u2·v2ᵀ ;  x = β·Âᵀy + z ;  w = α·Â·x
 *
 * Reproduces the gemver stages of examples/gemver-chain: Rank2Update (components.hpp:85-97), GemvTPartial
 * (components.hpp:142-167), ColReduce<true> (components.hpp:192-219) and Gemv (components.hpp:237-265), as wired by
 * the Gemver System (systems.hpp:71-133), in ONE persistent launch. The host double-precision reference is
 * gemver_chain::reference_chain's gemver lambda (common/chain_data.hpp:104-117).
 *
 * A is row-major n×n with row stride lda elements, stored as f32 or bf16 (a_dtype). Â is computed in f32 as
 * (a + u1[i]·v1[j]) + u2[i]·v2[j] with each operation rounded separately (no fused multiply-add), and written to B
 * (row stride ldb) when B is not NULL. Âᵀy is accumulated in f64 and combined in a fixed order; Â·x in f32 with a
 * fixed reduction tree: results do not depend on the launch shape or on other work on the GPU. z may be NULL (zero).
 * The default schedule is three streaming passes with grid barriers (cooperative launch); flags = CSPB_GEMVER_PANEL
 * pipelines column panels instead, so that the second read of each panel of Â hits L2 (HBM traffic: A once, Â once).
 * flags = CSPB_GEMVER_BULK runs the three passes with the matrix streamed through a shared-memory ring by bulk
 * asynchronous copies (one CTA per SM: 8 consumer warps and a producer warp); it applies when n is a multiple of 4
 * (f32) or 8 (bf16), the row strides are multiples of 16 bytes and every pointer is 16-byte aligned, and otherwise
 * falls back to the default. All schedules give bit-identical results.
 * ================================================================================================================== */
#define CSPB_GEMVER_PANEL 1
#define CSPB_GEMVER_BULK 2
/* flags = CSPB_GEMVER_LOWRANK with B == NULL: x and w are formed from A with the rank-2 update applied as four dot
 * products, x = β·(Aᵀy + v1(u1·y) + v2(u2·y)) + z and w = α·(A·x + u1(v1·x) + u2(v2·x)), in two streaming passes with
 * no per-element update. With B requested and a CSPB_BF16 matrix, pass 1 forms and stores Â and x comes from its
 * column sums as in the other schedules; only w takes the low-rank form (pass 2 re-reads the 16-bit A instead of
 * forming Â again). Other rounding than the schedules that form Â (within the f64 tolerance, not the same bits);
 * ignored for an f32 matrix with B. No counterpart in the reference, whose GEMVER always forms B. */
#define CSPB_GEMVER_LOWRANK 4
/* bits 8..15 of flags: the panel schedule's lag (pass 2 over a panel follows pass 1 over it by this many panels);
 * 0 = automatic (the panels the blocks in flight hold, plus one). A tuning knob: results do not depend on it. */
#define CSPB_GEMVER_LAG_MASK 0xff00
typedef struct cspb_gemver_desc {
    int64_t n;         /* rows = columns, >= 1 */
    int64_t lda;       /* row stride of A in elements, >= n */
    int64_t ldb;       /* row stride of B in elements, >= n (ignored when B is NULL) */
    int32_t a_dtype;   /* CSPB_F32 or CSPB_BF16 */
    int32_t flags;     /* reserved, 0 */
    const void* A;
    const float* u1;
    const float* v1;
    const float* u2;
    const float* v2;
    const float* y;
    const float* z;    /* may be NULL */
    float alpha;
    float beta;
    float* B;          /* may be NULL: Â is not materialized */
    float* x;          /* n */
    float* w;          /* n */
    void* workspace;
    size_t workspace_bytes;
} cspb_gemver_desc;

size_t cspb_gemver_workspace_bytes(int64_t n);
int cspb_gemver_fused(const cspb_gemver_desc* d, void* stream);

/* ONE GEMVER split by rows across GPUs (one process per GPU). The reference runs a GEMVER on one device only; this
 * splits its stages (examples/gemver-chain/components.hpp:85-97 Rank2Update, :142-167 GemvTPartial, :176-220
 * ColReduce, :227-266 Gemv) at the one place that needs every row: ColReduce's sum over row strips. A shard holds
 * rows [r0, r0 + rows) of A, B, u1, u2, y and w, and all n entries of v1, v2, z and x:
 *   cspb_gemver_rows_partial  Â rows (stored when B is not NULL) and colsum[j] = Σ_{i in shard} Â[i][j]·y[i] (f64, n)
 *   (the caller exchanges colsum and adds the shards' values in rank order: the same total on every rank)
 *   cspb_gemver_rows_finish   x = float(z + β·total) over all n columns, then w = α·Â·x over the shard's rows
 * A, B, u1, u2, y and w point at the shard's first row. flags must be 0. Each call is one cooperative launch on the
 * caller's stream; the workspace (cspb_gemver_rows_workspace_bytes) may be shared by the two calls of a shard. With
 * one shard (rows = n) the results equal cspb_gemver_fused's within rounding of the column sums' grouping. */
typedef struct cspb_gemver_rows_desc {
    int64_t n;         /* columns: the whole GEMVER's size, >= 1 */
    int64_t rows;      /* this shard's rows, 1 <= rows <= n */
    int64_t lda;       /* row stride of A in elements, >= n */
    int64_t ldb;       /* row stride of B in elements, >= n (ignored when B is NULL) */
    int32_t a_dtype;   /* CSPB_F32 or CSPB_BF16 */
    int32_t flags;     /* 0 */
    const void* A;     /* rows × n */
    const float* u1;   /* rows */
    const float* v1;   /* n */
    const float* u2;   /* rows */
    const float* v2;   /* n */
    const float* y;    /* rows */
    const float* z;    /* n, may be NULL */
    float alpha;
    float beta;
    float* B;          /* rows × n, may be NULL */
    float* x;          /* n: written by the finish */
    float* w;          /* rows: written by the finish */
    void* workspace;
    size_t workspace_bytes;
} cspb_gemver_rows_desc;

size_t cspb_gemver_rows_workspace_bytes(int64_t n, int64_t rows);
int cspb_gemver_rows_partial(const cspb_gemver_rows_desc* d, double* colsum, void* stream);
int cspb_gemver_rows_finish(const cspb_gemver_rows_desc* d, const double* colsum_total, void* stream);

/* ==================================================================================================================
 * BiCGK:  q = B·p ;  s = Bᵀ·r   (one pass over B)
 *
 * Reproduces Bicgk (examples/gemver-chain/systems.hpp:138-212): BicgkOnePass + RowReduce + ColReduce<false>
 * (components.hpp:277-358), and the q / s loops of reference_chain (common/chain_data.hpp:122-134). Bᵀr is
 * accumulated in f64, B·p in f32 with a fixed tree.
 * ================================================================================================================== */
typedef struct cspb_bicgk_desc {
    int64_t n;
    int64_t ldb;
    int32_t b_dtype;   /* CSPB_F32 or CSPB_BF16 */
    int32_t flags;     /* reserved, 0 */
    const void* B;
    const float* p;
    const float* r;
    float* q;
    float* s;
    void* workspace;
    size_t workspace_bytes;
} cspb_bicgk_desc;

size_t cspb_bicgk_workspace_bytes(int64_t n);
int cspb_bicgk_fused(const cspb_bicgk_desc* d, void* stream);

/* ==================================================================================================================
 * The gemver chain G1 → BiCGK → G2 in one persistent launch (examples/gemver-chain, Chain System systems.hpp:214-266;
 * host reference reference_chain common/chain_data.hpp:93-144):
 *   G1:    B1 = A0 + u1a·v1aᵀ + u2a·v2aᵀ,  x1 = β·B1ᵀ·ya + za,  w1 = α·B1·x1
 *   BiCGK: q = B1·x1,  s = B1ᵀ·w1
 *   G2:    B2 = B1 + u1b·v1bᵀ + u2b·v2bᵀ,  x2 = β·B2ᵀ·q + s,   w2 = α·B2·x2
 * Six passes over n² elements (the reference's nominal traffic counts eight). B1 and B2 may not be NULL.
 * ================================================================================================================== */
typedef struct cspb_chain_desc {
    int64_t n;
    const float* A0;                               /* n×n, row stride n */
    const float *u1a, *v1a, *u2a, *v2a, *ya, *za;  /* G1's vectors */
    const float *u1b, *v1b, *u2b, *v2b;            /* G2's rank-2 update */
    float alpha;                                   /* both GEMVERs (the reference ties one scale: 1/sqrt(n)) */
    float beta;
    float *B1, *x1, *w1, *q, *s, *B2, *x2, *w2;
    void* workspace;
    size_t workspace_bytes;
} cspb_chain_desc;

size_t cspb_chain_workspace_bytes(int64_t n);
int cspb_gemver_chain(const cspb_chain_desc* d, void* stream);

/* ==================================================================================================================
 * Ragged batch of independent GEMVERs in ONE persistent launch.
 *
 * Instance k has size n[k] (1 <= n[k] <= 65536). Its matrix starts at element a_off[k] of A (row stride
 * ld[k] = n[k] rounded up to a multiple of 8, so every row starts on a 16-byte boundary for both dtypes) and its
 * vectors at element v_off[k] of each packed vector array. The offsets are computed ON THE DEVICE from n[] by the
 * decoupled-lookback scan (cspb_exclusive_scan_u64) inside the call and written to a_off / v_off (count + 1 entries
 * each; the last is the total). max_elems / max_vec are the capacities of A (and B) and of each vector array; the
 * kernel checks the device-computed totals against them before touching memory and sets CSPB_DEV_CAPACITY when they
 * do not fit (an invalid n[k] sets CSPB_DEV_NEGATIVE). Per-instance alpha[k], beta[k] are device arrays.
 * `tune` holds 2 bits per size bucket (n < 512, < 1024, < 2048, >= 2048) choosing the tile geometry of that bucket
 * (0: 8 warps as 2 × 4, 1: 1 × 8, 2: 4 × 2); results depend only on (n, dtype, these bits), never on the rest of the
 * batch. Bits 8..9 set the work items a block takes per grab (0: 4, 1: 1, 2: 2, 3: 8) and bits 10..11 the blocks per
 * SM (0: as many as fit, 1: one fewer, 2: two, 3: one); neither changes a result.
 * Replaces the per-request launches a caller of the gemver example would make; ragged offsets follow
 * cs::ragged::counts_from (cospanmdao/include/naga/cospan/shape_hook.hpp:215-348) with u64 element offsets, since
 * 4096 instances of n up to 4096 overflow the reference's 32-bit offsets (device_scan.hpp:20-23).
 * ================================================================================================================== */
typedef struct cspb_gemver_batched_desc {
    int64_t count;          /* instances, >= 1 */
    int64_t max_elems;      /* capacity of A and B in elements */
    int64_t max_vec;        /* capacity of each packed vector array in elements */
    int32_t a_dtype;        /* CSPB_F32 or CSPB_BF16 */
    int32_t tune;           /* tile configuration index, 0 = default */
    const uint32_t* n;      /* device, count */
    const void* A;
    const float *u1, *v1, *u2, *v2, *y, *z;  /* packed; z may be NULL */
    const float* alpha;     /* device, count */
    const float* beta;      /* device, count */
    float* B;               /* may be NULL */
    float* x;
    float* w;
    uint64_t* a_off;        /* device out, count + 1 */
    uint64_t* v_off;        /* device out, count + 1 */
    void* workspace;
    size_t workspace_bytes;
} cspb_gemver_batched_desc;

size_t cspb_gemver_batched_workspace_bytes(int64_t count, int64_t max_elems, int64_t max_vec);
int cspb_gemver_batched(const cspb_gemver_batched_desc* d, void* stream);
/* Number of values `tune` may take (words with a bucket code of 3 are rejected). */
int cspb_gemver_batched_tunings(void);

/* The same launch over independent GEMVERs that live anywhere (a serving loop's resident models): a DEVICE array of
 * task descriptors instead of the packed layout. max_elems bounds Σ n·n and max_vec Σ n over the tasks (they size the
 * workspace: cspb_gemver_batched_workspace_bytes(count, max_elems, max_vec)). Per-task results are bit-identical to
 * cspb_gemver_fused on the same task (the same tile geometry at tune 0, the same reduction order). */
typedef struct cspb_gemver_task {
    int64_t n;
    int64_t lda;
    int64_t ldb;
    const void* A;           /* the call's a_dtype */
    float* B;                /* may be NULL */
    const float *u1, *v1, *u2, *v2, *y, *z;  /* z may be NULL */
    float* x;
    float* w;
    float alpha;
    float beta;
} cspb_gemver_task;

/* tune | CSPB_BATCH_LOWRANK (both batched entry points): an instance or task without B takes the low-rank form of
 * cspb_gemver_fused with CSPB_GEMVER_LOWRANK (the rank-2 update as dot products in the finishes); instances with B
 * are unchanged. */
#define CSPB_BATCH_LOWRANK (1 << 16)
/* tune | CSPB_BATCH_LOWRANK | CSPB_BATCH_NO_B (cspb_gemver_tasks, bf16 A): the caller states that no task has B. The
 * launch then uses a kernel variant without the paths that form and store Â, at 3 blocks per SM instead of 2; results
 * are bit-identical. A task with B under this flag sets CSPB_DEV_ARGUMENT: the call fails (its x and w are not valid)
 * and no B is written. A packed batch (cspb_gemver_batched) with B == NULL and a bf16 A takes that variant without
 * the flag. */
#define CSPB_BATCH_NO_B (1 << 17)
int cspb_gemver_tasks(const cspb_gemver_task* tasks, int64_t count, int64_t max_elems, int64_t max_vec,
                      int32_t a_dtype, int32_t tune, void* workspace, size_t workspace_bytes, void* stream);

/* ==================================================================================================================
 * NS residual, compressible (the reference's examples/ns-residual): one evaluation of R = -div F_conv + div F_visc
 * per cell plus the diagnostics, in ONE kernel whose face fluxes stay on chip.
 *
 * Reproduces NsFused (examples/ns-residual/systems.hpp:88-140) and hw_forward (handwritten.hpp:51-191): physics.hpp
 * (to_prim, grad_cell, hllc, visc_flux, cell_diag, MinMod / VanLeer), tile.hpp:39-229 (tile stages, face ownership),
 * components.hpp:393-628 (atomic diagnostics, deterministic reductions, error stage). The host double-precision
 * reference is reference_residual (reference.hpp:30-130).
 *
 * U and R are (4, ny, nx) f32, row-major. diag (device, 18 floats) receives, in this order:
 *   [0] Dt  [1] Ws  [2..5] Sq0..3           the atomic diagnostics (float atomics; Sq is order dependent)
 *   [6..9] detn.Det  [10] detd.Det  [11] detw.Det   the deterministic ones (f64 sums in a fixed order, rounded)
 *   [12..17] err.Err = atomic - deterministic: [dt, ws, sq0..sq3]
 * det_sq64 (device, 4 doubles, may be NULL) receives the f64 sums of R² before rounding.
 * ================================================================================================================== */
/* flags = CSPB_NS_REFERENCE_ROUNDING: the reference's formulas in their written order with every multiply and add
 * rounded separately (no fused multiply-add) and IEEE division and square root, so that R, min dt and max wave speed are
 * bit-identical to a sequential f32 evaluation of physics.hpp. The default (flags = 0) uses fused multiply-adds and
 * approximate reciprocals, divisions and reciprocal square roots in the face fluxes: faster, as close to the f64
 * reference, not the same bits. */
#define CSPB_NS_REFERENCE_ROUNDING 1
typedef struct cspb_ns_comp_desc {
    int32_t nx, ny;      /* >= 4 each */
    int32_t limiter;     /* 0 minmod, 1 van Leer */
    int32_t walls;       /* 1: no-slip adiabatic walls in y; 0: periodic in y. x is always periodic. */
    int32_t flags;       /* 0 or CSPB_NS_REFERENCE_ROUNDING */
    int32_t reserved;    /* 0 */
    const float* U;
    float* R;
    float* diag;         /* 18 floats */
    double* det_sq64;    /* 4 doubles, may be NULL */
    void* workspace;
    size_t workspace_bytes;
} cspb_ns_comp_desc;

size_t cspb_ns_comp_workspace_bytes(int32_t nx, int32_t ny);
int cspb_ns_compressible(const cspb_ns_comp_desc* d, void* stream);

/* One y-slab of a larger compressible grid (one process per GPU): rows [r0, r0 + rows) of U, rows >= 2. An edge whose
 * bit is set in `edges` is interior: bit 1, below the slab's row 0, reads the two rows r0 - 2, r0 - 1 of every field
 * from halo_lo; bit 2, above its last row, reads r0 + rows, r0 + rows + 1 from halo_hi; both are (4, 2, nx) f32,
 * the neighbouring slabs' rows (wrapped over the whole grid when it is periodic). An edge whose bit is clear takes the
 * whole grid's boundary rule there: the walls' mirror for the grid's first and last slab, or, with one slab, the
 * periodic wrap. R over the slab's cells is bit-identical to cspb_ns_compressible's rows of the whole grid, and so are
 * the per-cell dt and wave speed; diag and det_sq64 hold this slab's diagnostics (its min dt, max wave speed and
 * squared sums), which the caller combines across slabs in a fixed order (min, max, sum). The reference runs its
 * residual on one device (no counterpart); the exchange this implies is the 2-cell halo of its tiles
 * (examples/ns-residual/tile.hpp:39-49) across slabs, 2 rows x 4 fields per neighbour. */
typedef struct cspb_ns_comp_slab_desc {
    int32_t nx, rows;    /* nx >= 4, rows >= 2 */
    int32_t limiter;     /* 0 minmod, 1 van Leer */
    int32_t walls;       /* the whole grid's boundary rule in y: 1 walls, 0 periodic */
    int32_t flags;       /* 0 or CSPB_NS_REFERENCE_ROUNDING */
    int32_t edges;       /* bit 1: the edge below row 0 is interior; bit 2: the edge above row rows - 1 */
    const float* U;      /* (4, rows, nx) */
    const float* halo_lo;  /* (4, 2, nx) when edges & 1 */
    const float* halo_hi;  /* (4, 2, nx) when edges & 2 */
    float* R;            /* (4, rows, nx) */
    float* diag;         /* 18 floats, as cspb_ns_compressible, over this slab's cells */
    double* det_sq64;    /* 4 doubles, may be NULL */
    void* workspace;
    size_t workspace_bytes;
} cspb_ns_comp_slab_desc;

size_t cspb_ns_comp_slab_workspace_bytes(int32_t nx, int32_t rows);
int cspb_ns_comp_slab(const cspb_ns_comp_slab_desc* d, void* stream);

/* The reference's initial field (examples/ns-residual/physics.hpp:203-215, make_init main.cpp:100-112) on the
 * device: U(v, j, i) for amplitude amp. */
int cspb_ns_init_cons(float* U, int32_t nx, int32_t ny, float amp, void* stream);

/* ==================================================================================================================
 * NS residual, incompressible, 2D periodic collocated grid (no reference code computes it; the formula is
 *   r_u = u·∂u/∂x + v·∂u/∂y + ∂p/∂x − ν∇²u,   r_v = u·∂v/∂x + v·∂v/∂y + ∂p/∂y − ν∇²v,   r_c = ∂u/∂x + ∂v/∂y
 * with 2nd-order central differences on spacing h). u, v, p are (ny, nx) in f32 or bf16 storage; r_u, r_v, r_c are
 * f32. norms (device, 3 doubles, may be NULL) receives ||r_u||₂, ||r_v||₂, ||r_c||₂ from f64 sums in a fixed order.
 * CSPB_ERR_TOO_LARGE when the grid would need more than 2^31 − 1 tiles (blocks of 128 × 32 cells in f32 storage,
 * 512 × 16 in bf16).
 * ================================================================================================================== */
typedef struct cspb_ns_incomp_desc {
    int32_t nx, ny;      /* >= 3 each */
    int32_t dtype;       /* storage of u, v, p: CSPB_F32 or CSPB_BF16 */
    int32_t flags;       /* reserved, 0 */
    double h;
    double nu;
    const void* u;
    const void* v;
    const void* p;
    float* ru;
    float* rv;
    float* rc;
    double* norms;       /* 3 doubles, may be NULL */
    void* workspace;
    size_t workspace_bytes;
} cspb_ns_incomp_desc;

size_t cspb_ns_incomp_workspace_bytes(int32_t nx, int32_t ny);
int cspb_ns_incompressible(const cspb_ns_incomp_desc* d, void* stream);

/* One y-slab of a larger periodic grid (one process per GPU): rows [r0, r0 + rows) of u, v, p, with the row above
 * (r0 - 1) and the row below (r0 + rows), wrapped over the whole grid, passed as `up` and `dn` (nx floats of u, v, p
 * each) instead of being read from the slab. The residual rows are bit-identical to cspb_ns_incompressible's on the
 * whole grid; `sums` receives the slab's squared sums Σ r_u², Σ r_v², Σ r_c² (f64, 3), which the caller adds across
 * slabs in a fixed order before taking the roots. f32 storage, nx % 4 == 0, every pointer 16-byte aligned; flags
 * must be 0. The reference runs its residual on one device only (no counterpart); the exchange it implies is the
 * one-row halo of each slab. */
typedef struct cspb_ns_incomp_slab_desc {
    int32_t nx, rows;    /* nx >= 3, rows >= 1 */
    int32_t dtype;       /* CSPB_F32 */
    int32_t flags;       /* 0 */
    double h;
    double nu;
    const float* u;      /* rows × nx */
    const float* v;
    const float* p;
    const float* up[3];  /* the row above the slab: u, v, p */
    const float* dn[3];  /* the row below the slab: u, v, p */
    float* ru;           /* rows × nx */
    float* rv;
    float* rc;
    double* sums;        /* 3 doubles: the slab's squared sums */
    void* workspace;
    size_t workspace_bytes;
} cspb_ns_incomp_slab_desc;

size_t cspb_ns_incomp_slab_workspace_bytes(int32_t nx, int32_t rows);
int cspb_ns_incomp_slab(const cspb_ns_incomp_slab_desc* d, void* stream);

/* Many incompressible residuals (any sizes, one storage dtype) in ONE persistent launch, from a DEVICE array of task
 * descriptors. max_cells bounds Σ nx·ny (it sizes the workspace). Per-task results, norms included, are bit-identical
 * to cspb_ns_incompressible on the same task (the same decomposition, the same reduction order). */
typedef struct cspb_ns_incomp_task {
    int32_t nx, ny;
    double h;
    double nu;
    const void* u;
    const void* v;
    const void* p;
    float* ru;
    float* rv;
    float* rc;
    double* norms;       /* 3 doubles, may be NULL */
} cspb_ns_incomp_task;

size_t cspb_ns_incomp_tasks_workspace_bytes(int64_t count, int64_t max_cells);
int cspb_ns_incomp_tasks(const cspb_ns_incomp_task* tasks, int64_t count, int64_t max_cells, int32_t dtype,
                         void* workspace, size_t workspace_bytes, void* stream);

/* ==================================================================================================================
 * Device scan: out[0..n] = the exclusive scan of in[0..n), out[n] = the total, in ONE single-pass launch
 * (decoupled lookback). The u32 variant wraps mod 2^32 like cs::detail::exclusive_scan_u32
 * (cospanmdao/include/naga/cospan/device_scan.hpp:46-110), which it replaces bit for bit; the u64 variant wraps
 * mod 2^64. in and out must not overlap. n == 0 writes out[0] = 0.
 * ================================================================================================================== */
size_t cspb_scan_workspace_bytes(int64_t n);
int cspb_exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, void* workspace, size_t workspace_bytes,
                            void* stream);
int cspb_exclusive_scan_u64(const uint64_t* in, uint64_t* out, int64_t n, void* workspace, size_t workspace_bytes,
                            void* stream);

/* ==================================================================================================================
 * A ragged column from an integer variable (cs::detail::build_column, cospanmdao/include/naga/cospan/
 * shape_hook.hpp:215-348): counts mode (offsets_mode = 0) reads count values src[i * k] (column 0 of a rank-2 [N, k]
 * source, k = 1 for rank 1), writes extents[i] = max(value, 0) narrowed to u32 and offs = their exclusive scan
 * (count + 1 entries); offsets mode (offsets_mode = 1) reads count = N + 1 offsets, writes offs = the values and
 * extents[i] = offs[i+1] - offs[i]. The flag bits follow the reference: 1 = a negative value, offs[0] != 0 or a
 * decrease; 2 = a value or a total past 2^32 - 1; 4 (CSPB_COLUMN_TIMEOUT, no counterpart in the reference) = the
 * bounded look-back of the scan gave up and the offsets are not valid. total_flag (device or mapped host memory,
 * 2 words) receives [offs[N], flag]. Single pass: narrow + scan + wrap check in one launch.
 * ================================================================================================================== */
int cspb_build_column(const void* src, int32_t src_dtype, int64_t count, int64_t k, int32_t offsets_mode,
                      uint32_t* extents, uint32_t* offs, uint32_t* total_flag, void* workspace,
                      size_t workspace_bytes, void* stream);

/* The same column with 64-bit offsets (offs: count + 1 u64 in counts mode, N + 1 in offsets mode), for a ragged
 * variable whose total may pass 2^32 - 1: the runtime's opt-in u64 offset type (cs::ragged::counts_from<uint64_t>),
 * which the reference's roadmap names as the next step for its u32-only columns (internal/ROADMAP.md:106; today
 * shape_hook.hpp:455-457 rejects such totals). Each extent is still a u32: flag 2 marks a single value or offset
 * difference past 2^32 - 1, never the total. total_flag (2 u64) receives [offs[N], flag], the flag word holding the
 * same bits as cspb_build_column's total_flag[1]. */
int cspb_build_column64(const void* src, int32_t src_dtype, int64_t count, int64_t k, int32_t offsets_mode,
                        uint32_t* extents, uint64_t* offs, uint64_t* total_flag, void* workspace,
                        size_t workspace_bytes, void* stream);

/* ==================================================================================================================
 * cspb_build_column_static: cspb_build_column with no workspace argument, for callers that cannot allocate device
 * memory at the call site (a foreign-language binding that holds only the column's pointers and no allocator, code
 * running where an allocation would stall or be refused). It allocates nothing: its scratch is a fixed 131,328-byte array
 * in the library's device image (one per device), looked up in the current device's context by each call;
 * make the first call on a device before any stream capture begins. Results are bit-identical to cspb_build_column.
 * Limit: at most CSPB_BUILD_COLUMN_STATIC_MAX extents (count in counts mode, count - 1 in offsets mode); larger inputs
 * return CSPB_ERR_TOO_LARGE before any device work. The scratch is shared by every call on a device, so calls on one
 * device must not overlap in time (same stream, or ordered by events); overlapping calls race on it. The device status
 * word of this call lives in that scratch, out of the caller's reach, so everything the device finds goes to the flag
 * word total_flag[1]: CSPB_COLUMN_NEGATIVE, CSPB_COLUMN_EXCEEDS32, and CSPB_COLUMN_TIMEOUT when the scan's bounded wait
 * gave up (offsets not valid). The scratch's device address is asked of the CUDA runtime on every call (a cached
 * address would outlive a cudaDeviceReset); the first call on a device also loads the library's device image there.
 * No counterpart in the reference (its build_column allocates its temporaries on every call).
 * ================================================================================================================== */
#define CSPB_BUILD_COLUMN_STATIC_MAX (1 << 24)
int cspb_build_column_static(const void* src, int32_t src_dtype, int64_t count, int64_t k, int32_t offsets_mode,
                             uint32_t* extents, uint32_t* offs, uint32_t* total_flag, void* stream);

/* ==================================================================================================================
 * Seeded inputs on the device: the reference's generator gemver_chain::hash_unit (common/chain_data.hpp:34-49).
 * dist 0: hash_unit(seed, i) in [-1, 1); dist 1: (hash_unit(seed, i) + 1) / 2 in [0, 1), exactly (h >> 8) · 2^-24.
 * out_dtype CSPB_F32 or CSPB_BF16 (round to nearest even). Element i of the output is at out + i (index_base added to
 * i for the hash).
 * ================================================================================================================== */
int cspb_fill_hash(void* out, int32_t out_dtype, int64_t count, uint64_t index_base, uint32_t seed, int32_t dist,
                   void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CSPB_H */
