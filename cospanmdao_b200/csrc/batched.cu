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
//      pass-1 unit of an instance forms its x (fixed order) and publishes a flag; a pass-2 unit waits (bounded) for
//      its instance's flag. A waiting block only ever waits on work that running blocks hold and that never waits
//      itself, so the launch needs no co-residency guarantee.
// Per-instance results do not depend on the rest of the batch: the geometry is a function of (n, dtype, tuning) and
// every reduction runs in a fixed order (rowpass.cuh).
#include "rowpass.cuh"

namespace cspb {
namespace batch {

constexpr int kThreads = kPassThreads;
constexpr int kSets = 6;  // a, v, p, w, s, u
enum { SA = 0, SV = 1, SP = 2, SW = 3, SS = 4, SU = 5 };

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
    uint32_t tune;
    int bf16;
    uint64_t* sizes;  // [kSets][count]
    uint8_t* wx;      // [count]
    uint32_t* ctrl;
};

__global__ void k_plan(PlanK g) {
    for (int64_t k = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; k < g.count; k += int64_t(gridDim.x) * blockDim.x) {
        uint32_t n = g.n[k];
        if (n < 1 || n > 65536) {
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
    }
}

struct RunK {
    int64_t count;
    const uint32_t* n;
    const uint8_t* wx;
    const uint64_t* off[kSets];  // each count + 1
    uint64_t cap[kSets - 1];     // capacities of a, v, p, w, s (elements)
    const void* A;
    const float *u1, *v1, *u2, *v2, *y, *z, *alpha, *beta;
    float *B, *x, *w;
    double* P;
    float* Wp;
    uint32_t* strip_done;
    uint32_t* p1_done;   // [count]
    uint32_t* x_ready;   // [count]
    uint32_t* ctrl;
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

template <typename T>
__device__ __forceinline__ PassArgs instance_args(const RunK& g, int64_t k, int wx, bool bf16) {
    PassArgs a{};
    const uint32_t n = g.n[k];
    const uint64_t ld = (uint64_t(n) + 7) / 8 * 8;
    const uint64_t ao = __ldcg(g.off[SA] + k), vo = __ldcg(g.off[SV] + k);
    a.n = n;
    a.src = static_cast<const T*>(g.A) + ao;
    a.lds = int64_t(ld);
    a.dst = g.B ? g.B + ao : nullptr;
    a.ldd = int64_t(ld);
    a.u1 = g.u1 + vo; a.v1 = g.v1 + vo; a.u2 = g.u2 + vo; a.v2 = g.v2 + vo;
    a.cyB = g.y + vo;
    a.PB = g.P + __ldcg(g.off[SP] + k);
    a.xv = g.x + vo;
    a.Wp = g.Wp + __ldcg(g.off[SW] + k);
    a.strip_done = g.strip_done + __ldcg(g.off[SS] + k);
    a.rout1 = g.w + vo;
    a.rscale1 = g.alpha[k];
    const int64_t S = rows_of(wx), CW = cols_of(wx, bf16);
    a.strips = (n + S - 1) / S;
    a.chunks = (n + CW - 1) / CW;
    return a;
}

// x of one instance by one block: x[j] = z[j] + β · Σ_s P[s][j], strips in order (f64), then rounded.
__device__ __forceinline__ void instance_x(const PassArgs& a, const float* z, float beta, float* x) {
    for (int64_t j = threadIdx.x; j < a.n; j += blockDim.x) {
        double s = 0.0;
        for (int64_t st = 0; st < a.strips; ++st) s += __ldcg(a.PB + st * a.n + j);
        const double zz = z ? double(__ldcg(z + j)) : 0.0;
        x[j] = float(zz + double(beta) * s);
    }
}

template <typename T, int WX>
__device__ __forceinline__ void unit1(const PassArgs& a, int64_t unit, unsigned char* smem) {
    pass_unit<T, WX, true, true, false, true, false>(a, unit, true, smem);
}
template <typename T, int WX, bool FROM_B>
__device__ __forceinline__ void unit2(const PassArgs& a, int64_t unit, unsigned char* smem) {
    if constexpr (FROM_B) {
        PassArgs b = a;
        b.src = a.dst;
        b.lds = a.ldd;
        pass_unit<float, WX, false, false, false, false, true>(b, unit, true, smem);
    } else {
        pass_unit<T, WX, true, true, false, false, true>(a, unit, true, smem);
    }
}

template <typename T, bool FROM_B>
__global__ void __launch_bounds__(kThreads, 2) k_run(RunK g) {
    constexpr bool bf16 = sizeof(T) == 2;
    __shared__ __align__(16) unsigned char smem[pass_smem_bytes<T, 1>() > pass_smem_bytes<T, 4>()
                                                    ? pass_smem_bytes<T, 1>()
                                                    : pass_smem_bytes<T, 4>()];
    // the device-computed totals must fit the capacities the caller declared (decided by one thread, so the whole
    // block leaves together)
    const uint64_t U1 = __ldcg(g.off[SU] + g.count);
    __shared__ int s_go;
    if (threadIdx.x == 0) {
        bool fits = 2 * U1 < 0xffffffffull;
        for (int s = 0; s < kSets - 1; ++s) fits = fits && __ldcg(g.off[s] + g.count) <= g.cap[s];
        if (!fits) set_status(g.ctrl, CSPB_DEV_CAPACITY);
        s_go = fits && !status_bad(g.ctrl);  // status set by the plan: an invalid size
    }
    __syncthreads();
    if (!s_go) return;
    __shared__ int s_last;
    for (;;) {
        const uint32_t item32 = grab_work(g.ctrl, kWork0);
        const uint64_t item = item32;
        if (item >= 2 * U1) break;
        const bool pass2 = item >= U1;
        const uint64_t u = pass2 ? item - U1 : item;
        const int64_t k = find_instance(g.off[SU], g.count, u);
        const int64_t unit = int64_t(u - __ldcg(g.off[SU] + k));
        const int wx = g.wx[k];
        const PassArgs a = instance_args<T>(g, k, wx, bf16);
        if (!pass2) {
            switch (wx) {
                case 1: unit1<T, 1>(a, unit, smem); break;
                case 4: unit1<T, 4>(a, unit, smem); break;
                default: unit1<T, 2>(a, unit, smem); break;
            }
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) s_last = atomicAdd(g.p1_done + k, 1u) == uint32_t(a.strips * a.chunks - 1);
            __syncthreads();
            if (s_last) {
                __threadfence();
                const uint64_t vo = __ldcg(g.off[SV] + k);
                instance_x(a, g.z ? g.z + vo : nullptr, g.beta[k], g.x + vo);
                __threadfence();
                __syncthreads();
                if (threadIdx.x == 0) st_release(g.x_ready + k, 1u);
            }
        } else {
            __shared__ int s_ok;
            if (threadIdx.x == 0) s_ok = ld_acquire(g.x_ready + k) != 0u || wait_change(g.x_ready + k, 0u, g.ctrl);
            __syncthreads();
            if (!s_ok) break;
            __threadfence();
            switch (wx) {
                case 1: unit2<T, 1, FROM_B>(a, unit, smem); break;
                case 4: unit2<T, 4, FROM_B>(a, unit, smem); break;
                default: unit2<T, 2, FROM_B>(a, unit, smem); break;
            }
        }
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
    uint64_t capP = 0, capW = 0, capS = 0;
};

BatchLayout batch_layout(int64_t count, int64_t max_elems, int64_t max_vec) {
    BatchLayout L;
    const uint64_t Smin = 64, CWmin = 128;  // the smallest strip and chunk of any tuning
    L.capP = uint64_t(max_elems) / Smin + uint64_t(max_vec);
    L.capW = uint64_t(max_elems) / CWmin + uint64_t(max_vec);
    L.capS = uint64_t(max_vec) / Smin + uint64_t(count);
    size_t o = kCtrlBytes;
    L.off_sizes = o;
    o = align_up(o + size_t(batch::kSets) * size_t(count) * 8, 256);
    L.off_offs = o;  // p, w, s, u offsets (a and v go to the caller)
    o = align_up(o + 4 * size_t(count + 1) * 8, 256);
    L.off_wx = o;
    o = align_up(o + size_t(count), 256);
    L.off_p1 = o;  // p1_done then x_ready, zeroed together with the strip counters
    o = align_up(o + size_t(count) * 4, 256);
    L.off_xr = o;
    o = align_up(o + size_t(count) * 4, 256);
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

int cspb_gemver_batched_tunings(void) { return 1 << 8; }

int cspb_gemver_batched(const cspb_gemver_batched_desc* d, void* stream) {
    if (!d) return CSPB_ERR_ARGUMENT;
    if (d->count < 1 || d->count > (int64_t(1) << 26) || d->max_elems < 1 || d->max_vec < 1) return CSPB_ERR_ARGUMENT;
    if (!d->n || !d->A || !d->u1 || !d->v1 || !d->u2 || !d->v2 || !d->y || !d->alpha || !d->beta || !d->x || !d->w ||
        !d->a_off || !d->v_off)
        return CSPB_ERR_ARGUMENT;
    if (d->a_dtype != CSPB_F32 && d->a_dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    if (d->tune < 0 || d->tune >= cspb_gemver_batched_tunings()) return CSPB_ERR_UNSUPPORTED;
    for (uint32_t b = 0; b < 4; ++b)
        if (((uint32_t(d->tune) >> (2 * b)) & 3u) == 3u) return CSPB_ERR_UNSUPPORTED;
    if (!aligned(d->A, 16) || (d->B && !aligned(d->B, 16))) return CSPB_ERR_ARGUMENT;
    const BatchLayout L = batch_layout(d->count, d->max_elems, d->max_vec);
    if (!d->workspace || !aligned(d->workspace, 256) || d->workspace_bytes < L.total) return CSPB_ERR_WORKSPACE;
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    char* ws = static_cast<char*>(d->workspace);
    const bool bf16 = d->a_dtype == CSPB_BF16;
    // control block, p1_done, x_ready, strip counters: one zeroing of the contiguous range
    if (cudaMemsetAsync(ws, 0, kCtrlBytes, st) != cudaSuccess) return CSPB_ERR_CUDA;
    if (cudaMemsetAsync(ws + L.off_p1, 0, L.off_scan - L.off_p1, st) != cudaSuccess) return CSPB_ERR_CUDA;

    batch::PlanK pk{};
    pk.count = d->count;
    pk.n = d->n;
    pk.tune = uint32_t(d->tune);
    pk.bf16 = bf16;
    pk.sizes = reinterpret_cast<uint64_t*>(ws + L.off_sizes);
    pk.wx = reinterpret_cast<uint8_t*>(ws + L.off_wx);
    pk.ctrl = reinterpret_cast<uint32_t*>(ws);
    int64_t pb = (d->count + 255) / 256;
    if (pb > 4096) pb = 4096;
    batch::k_plan<<<unsigned(pb), 256, 0, st>>>(pk);
    if (cudaGetLastError() != cudaSuccess) return CSPB_ERR_LAUNCH;

    uint64_t* offs = reinterpret_cast<uint64_t*>(ws + L.off_offs);
    uint64_t* outs[batch::kSets] = {d->a_off, d->v_off, offs, offs + (d->count + 1), offs + 2 * (d->count + 1),
                                    offs + 3 * (d->count + 1)};
    for (int s = 0; s < batch::kSets; ++s) {
        const int r = cspb_exclusive_scan_u64(pk.sizes + size_t(s) * size_t(d->count), outs[s], d->count,
                                              ws + L.off_scan, cspb_scan_workspace_bytes(d->count), stream);
        if (r != CSPB_OK) return r;
    }

    batch::RunK g{};
    g.count = d->count;
    g.n = d->n;
    g.wx = pk.wx;
    for (int s = 0; s < batch::kSets; ++s) g.off[s] = outs[s];
    g.cap[batch::SA] = uint64_t(d->max_elems);
    g.cap[batch::SV] = uint64_t(d->max_vec);
    g.cap[batch::SP] = L.capP;
    g.cap[batch::SW] = L.capW;
    g.cap[batch::SS] = L.capS;
    g.A = d->A;
    g.u1 = d->u1; g.v1 = d->v1; g.u2 = d->u2; g.v2 = d->v2; g.y = d->y; g.z = d->z;
    g.alpha = d->alpha;
    g.beta = d->beta;
    g.B = d->B;
    g.x = d->x;
    g.w = d->w;
    g.P = reinterpret_cast<double*>(ws + L.off_P);
    g.Wp = reinterpret_cast<float*>(ws + L.off_W);
    g.strip_done = reinterpret_cast<uint32_t*>(ws + L.off_S);
    g.p1_done = reinterpret_cast<uint32_t*>(ws + L.off_p1);
    g.x_ready = reinterpret_cast<uint32_t*>(ws + L.off_xr);
    g.ctrl = reinterpret_cast<uint32_t*>(ws);
    const void* kern;
    if (bf16) kern = reinterpret_cast<const void*>(batch::k_run<__nv_bfloat16, false>);
    else if (d->B) kern = reinterpret_cast<const void*>(batch::k_run<float, true>);
    else kern = reinterpret_cast<const void*>(batch::k_run<float, false>);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, batch::kThreads, 0) != cudaSuccess || per_sm < 1)
        return CSPB_ERR_LAUNCH;
    void* args[] = {&g};
    if (cudaLaunchKernel(kern, dim3(unsigned(per_sm * di.sms)), dim3(batch::kThreads), args, 0, st) != cudaSuccess)
        return CSPB_ERR_LAUNCH;
    return CSPB_OK;
}

}  // extern "C"
