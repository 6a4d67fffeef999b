// Pulse compaction for the download of a chunk's results.
//
// The pulse accumulator's output keeps max_calls slots a ZMW (the
// reference's BatchVectors layout); a chunk fills about a quarter of them.
// Before the results cross to the host the valid records are packed ZMW
// after ZMW: one exclusive scan of the counts (CUB) and a gather, a warp per
// ZMW moving its records as 4-byte words (coalesced).  The total goes to a
// mapped host word, one of two alternating slots, so a caller can size the
// copy of one call's records while the next call is queued.
#include <algorithm>
#include <string>

#include <cub/device/device_scan.cuh>

#include "hw_device.cuh"

using namespace hwk;

namespace {

__global__ void ClampKernel(const uint32_t* lens, uint32_t cap, uint32_t n, uint64_t* counts)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z == 0) counts[n] = 0;
    if (z < n) counts[z] = min(lens[z], cap);
}

__global__ void __launch_bounds__(256) GatherKernel(const hw_pulse* pulses, const uint64_t* offsets, uint32_t cap,
                                                    uint32_t n, hw_pulse* out, volatile uint64_t* total)
{
    constexpr uint32_t kWords = sizeof(hw_pulse) / 4;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    if (blockIdx.x == 0 && threadIdx.x == 0) *total = offsets[n];
    for (uint32_t z = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32; z < n; z += warps)
    {
        const uint64_t o = offsets[z];
        const uint32_t words = (uint32_t)(offsets[z + 1] - o) * kWords;
        const uint32_t* src = reinterpret_cast<const uint32_t*>(pulses + (size_t)z * cap);
        uint32_t* dst = reinterpret_cast<uint32_t*>(out + o);
        for (uint32_t w = lane; w < words; w += 32) dst[w] = src[w];
    }
}

int Fail(int code, const std::string& msg) { return hwk::SetLastError(code, msg.c_str()); }

}   // namespace

struct hw_pulse_compactor
{
    uint32_t numZmw = 0;
    void* scanTmp = nullptr;
    size_t scanBytes = 0;
    uint64_t* host = nullptr;        // mapped: the totals of alternate calls
    uint64_t* hostDev = nullptr;
    uint64_t calls = 0;
    ~hw_pulse_compactor() { cudaFree(scanTmp); cudaFreeHost(host); }
};

extern "C" {

int hw_pulse_compactor_create(uint32_t num_zmw, hw_pulse_compactor** out)
{
    if (!out || num_zmw == 0) return Fail(HW_ERR_INVALID_ARG, "hw_pulse_compactor_create: bad argument");
    *out = nullptr;
    auto h = new hw_pulse_compactor;
    h->numZmw = num_zmw;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, h->scanBytes, static_cast<uint64_t*>(nullptr),
                                                  static_cast<uint64_t*>(nullptr), (int)num_zmw + 1);
    if (e == cudaSuccess) e = cudaMalloc(&h->scanTmp, h->scanBytes);
    if (e == cudaSuccess) e = cudaHostAlloc((void**)&h->host, 2 * sizeof(uint64_t), cudaHostAllocMapped);
    if (e == cudaSuccess)
    {
        h->host[0] = h->host[1] = 0;   // pinned memory comes uninitialised
        e = cudaHostGetDevicePointer((void**)&h->hostDev, h->host, 0);
    }
    if (e != cudaSuccess)
    {
        delete h;
        return Fail(HW_ERR_CUDA, std::string("hw_pulse_compactor_create: ") + cudaGetErrorString(e));
    }
    *out = h;
    return HW_OK;
}

int hw_pulse_compactor_destroy(hw_pulse_compactor* h)
{
    delete h;
    return HW_OK;
}

int hw_pulses_compact(hw_pulse_compactor* h, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                      hw_pulse* d_out, uint64_t* d_offsets, uint32_t* slot, void* stream)
{
    if (!h || !d_pulses || !d_lens || !d_out || !d_offsets || max_calls == 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_pulses_compact: bad argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t n = h->numZmw, threads = 256;
    const uint32_t sl = (uint32_t)(h->calls & 1);
    ClampKernel<<<(n + threads) / threads, threads, 0, s>>>(d_lens, max_calls, n, d_offsets);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cub::DeviceScan::ExclusiveSum(h->scanTmp, h->scanBytes, d_offsets, d_offsets, (int)n + 1, s);
    if (e == cudaSuccess)
    {
        const uint32_t blocks = std::min<uint32_t>((n + 7) / 8, 148 * 8);
        GatherKernel<<<blocks, 256, 0, s>>>(d_pulses, d_offsets, max_calls, n, d_out, h->hostDev + sl);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_pulses_compact: ") + cudaGetErrorString(e));
    if (slot) *slot = sl;
    ++h->calls;
    return HW_OK;
}

int hw_pulse_compactor_total(const hw_pulse_compactor* h, uint32_t slot, uint64_t* total)
{
    if (!h || slot > 1 || !total) return Fail(HW_ERR_INVALID_ARG, "hw_pulse_compactor_total: bad argument");
    *total = ((volatile uint64_t*)h->host)[slot];
    return HW_OK;
}

}   // extern "C"
