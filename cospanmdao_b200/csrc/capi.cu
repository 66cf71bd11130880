// capi.cu — status strings, the status-word readback, device facts, and the seeded input generator.
#include <mutex>

#include "common.cuh"
#include "mbar.cuh"

namespace cspb_host {

DeviceInfo device_info() {
    // Cached per device: the attribute queries cost microseconds, a GEMVER at small n costs about as much.
    static std::mutex mu;
    static DeviceInfo cache[64];
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return DeviceInfo{};
    std::lock_guard<std::mutex> lock(mu);
    DeviceInfo& d = cache[dev];
    if (d.device != dev) {
        DeviceInfo fresh;
        fresh.device = dev;
        if (cudaDeviceGetAttribute(&fresh.sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&fresh.coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess)
            return DeviceInfo{};
        d = fresh;
    }
    return d;
}

int map_cuda_error(cudaError_t e) { return e == cudaSuccess ? CSPB_OK : CSPB_ERR_CUDA; }

namespace {
__global__ void k_clear_ctrl(uint32_t* ctrl) {
    asm volatile("griddepcontrol.launch_dependents;");  // the dependent grid may be scheduled from now on
    ctrl[threadIdx.x] = 0u;
}
}  // namespace

int clear_ctrl(void* ws, cudaStream_t st) {
    k_clear_ctrl<<<1, unsigned(cspb::kCtrlBytes / 4), 0, st>>>(static_cast<uint32_t*>(ws));
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

int launch_dependent(const void* kern, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void** args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelExC(&cfg, kern, args) == cudaSuccess) return CSPB_OK;
    // a driver that refuses the attribute: a plain launch, ordered after the previous kernel as usual
    (void)cudaGetLastError();
    return cudaLaunchKernel(kern, grid, block, args, smem, st) == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

}  // namespace cspb_host

namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

// The 24 hash bits of gemver_chain::hash_unit (examples/gemver-chain/common/chain_data.hpp:43-48).
__device__ __forceinline__ uint32_t hash24(uint32_t seed, uint64_t index) {
    const uint32_t lo = static_cast<uint32_t>(index);
    const uint32_t hi = static_cast<uint32_t>(index >> 32);
    const uint32_t h = mix32(mix32(seed * 0x9e3779b9u + 0x85ebca6bu) ^ mix32(lo + mix32(hi + seed)));
    return h >> 8;
}

template <typename T>
__global__ void k_fill_hash(T* out, int64_t count, uint64_t base, uint32_t seed, int dist) {
    const int64_t stride = int64_t(gridDim.x) * blockDim.x;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
        const uint32_t h = hash24(seed, base + uint64_t(i));
        // dist 0: h·2^-23 - 1 in [-1, 1) (exact in f32); dist 1: h·2^-24 in [0, 1)
        const float v = dist == 0 ? float(h) * (1.0f / 8388608.0f) - 1.0f : float(h) * (1.0f / 16777216.0f);
        if constexpr (sizeof(T) == 4) out[i] = v;
        else out[i] = __float2bfloat16_rn(v);
    }
}

}  // namespace

extern "C" {

const char* cspb_status_string(int status) {
    switch (status) {
        case CSPB_OK: return "ok";
        case CSPB_ERR_ARGUMENT: return "invalid argument";
        case CSPB_ERR_WORKSPACE: return "workspace missing, misaligned or too small";
        case CSPB_ERR_LAUNCH: return "kernel launch failed";
        case CSPB_ERR_TIMEOUT: return "a device-side wait timed out";
        case CSPB_ERR_NEGATIVE: return "a ragged count is negative or the offsets are invalid";
        case CSPB_ERR_EXCEEDS32: return "a ragged value or total is past 2^32 - 1";
        case CSPB_ERR_UNSUPPORTED: return "unsupported dtype or option";
        case CSPB_ERR_CUDA: return "CUDA runtime error";
        case CSPB_ERR_CAPACITY: return "device-computed totals exceed the declared capacities";
        case CSPB_ERR_TOO_LARGE: return "input larger than the fixed scratch allows (CSPB_BUILD_COLUMN_STATIC_MAX)";
        default: return "unknown status";
    }
}

const char* cspb_version(void) { return "cspb 0.1 sm_100a"; }

int cspb_read_status(const void* workspace, uint32_t* raw, void* stream) {
    if (!workspace) return CSPB_ERR_ARGUMENT;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint32_t word = 0;
    cudaError_t e = cudaMemcpyAsync(&word, workspace, sizeof(word), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return CSPB_ERR_CUDA;
    if (raw) *raw = word;
    if (word & CSPB_DEV_TIMEOUT) return CSPB_ERR_TIMEOUT;
    if (word & CSPB_DEV_NEGATIVE) return CSPB_ERR_NEGATIVE;
    if (word & CSPB_DEV_EXCEEDS32) return CSPB_ERR_EXCEEDS32;
    if (word & CSPB_DEV_CAPACITY) return CSPB_ERR_CAPACITY;
    if (word & CSPB_DEV_ARGUMENT) return CSPB_ERR_ARGUMENT;
    return CSPB_OK;
}

int cspb_fill_hash(void* out, int32_t out_dtype, int64_t count, uint64_t index_base, uint32_t seed, int32_t dist,
                   void* stream) {
    if (count < 0 || (count > 0 && !out) || (dist != 0 && dist != 1)) return CSPB_ERR_ARGUMENT;
    if (out_dtype != CSPB_F32 && out_dtype != CSPB_BF16) return CSPB_ERR_UNSUPPORTED;
    if (count == 0) return CSPB_OK;
    const cspb_host::DeviceInfo di = cspb_host::device_info();
    if (di.device < 0) return CSPB_ERR_CUDA;
    int64_t blocks = (count + 255) / 256;
    const int64_t cap = int64_t(di.sms) * 8;
    if (blocks > cap) blocks = cap;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (out_dtype == CSPB_F32)
        k_fill_hash<float><<<unsigned(blocks), 256, 0, st>>>(static_cast<float*>(out), count, index_base, seed, dist);
    else
        k_fill_hash<__nv_bfloat16><<<unsigned(blocks), 256, 0, st>>>(static_cast<__nv_bfloat16*>(out), count,
                                                                     index_base, seed, dist);
    return cudaGetLastError() == cudaSuccess ? CSPB_OK : CSPB_ERR_LAUNCH;
}

}  // extern "C"
