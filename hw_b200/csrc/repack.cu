// Ingest repacking for sm_100a: sensor packets -> TraceBatch chunks.
//
// Restates the data shuffle of appModules/BlockRepacker.cpp:200-345
// (BatchFiller::Process): every cache line of a packet block (32 int16 or 64
// uint8 ZMWs of one frame) lands at its ZMW's lane and frame of the pool's
// chunk [lanes][frames][64].
//
// The host turns the chunk's packet table into copy segments -- the overlap
// of one packet block with one lane, num_frames rows of 64 or 128 bytes with
// the block's and the lane's row strides -- and one kernel moves them: a
// 256-thread block per segment, 16-byte vector loads (streaming, the packets
// are read once) and stores.  The copy is pure HBM traffic: every byte read
// once and written once.
#include <algorithm>
#include <string>
#include <vector>

#include "hw_device.cuh"

using namespace hwk;

namespace {

struct RepackSeg
{
    uint64_t src, dst;            // device addresses of row 0
    uint32_t rows, vecsLog2;      // rows; 16-byte vectors per row = 1 << vecsLog2
    uint32_t srcStride, dstStride;  // bytes between rows
};

__global__ void __launch_bounds__(256) RepackKernel(const RepackSeg* segs)
{
    const RepackSeg sg = segs[blockIdx.x];
    const uint32_t vpr = 1u << sg.vecsLog2;
    const uint32_t n = sg.rows << sg.vecsLog2;
    const char* src = reinterpret_cast<const char*>(sg.src);
    char* dst = reinterpret_cast<char*>(sg.dst);
    for (uint32_t v = threadIdx.x; v < n; v += blockDim.x)
    {
        const uint32_t row = v >> sg.vecsLog2, col = (v & (vpr - 1)) * 16u;
        const uint4 x = __ldcs(reinterpret_cast<const uint4*>(src + (size_t)row * sg.srcStride + col));
        *reinterpret_cast<uint4*>(dst + (size_t)row * sg.dstStride + col) = x;
    }
}

int Fail(int code, const std::string& msg) { return hwk::SetLastError(code, msg.c_str()); }

}   // namespace

struct hw_repacker
{
    uint32_t numZmw = 0, lanesPerPool = 0, F = 0, elem = 2, pools = 0;
    std::vector<RepackSeg> host;
    RepackSeg* staging[2] = {nullptr, nullptr};   // pinned copies of the segment tables
    size_t stagingCap[2] = {0, 0};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool inFlight[2] = {false, false};
    RepackSeg* dev = nullptr;
    size_t devCap = 0;
    uint64_t calls = 0;
    ~hw_repacker()
    {
        for (int b = 0; b < 2; ++b)
        {
            if (ev[b]) { cudaEventSynchronize(ev[b]); cudaEventDestroy(ev[b]); }
            cudaFreeHost(staging[b]);
        }
        cudaFree(dev);
    }
};

extern "C" {

int hw_repacker_create(uint32_t num_zmw, uint32_t lanes_per_pool, uint32_t frames_per_chunk, int32_t encoding,
                       hw_repacker** out)
{
    if (!out || num_zmw == 0 || lanes_per_pool == 0 || frames_per_chunk == 0 || (encoding != 0 && encoding != 1))
        return Fail(HW_ERR_INVALID_ARG, "hw_repacker_create: bad argument");
    if (num_zmw % kLane != 0) return Fail(HW_ERR_INVALID_ARG, "hw_repacker_create: num_zmw must be a multiple of 64");
    *out = nullptr;
    auto r = new hw_repacker;
    r->numZmw = num_zmw;
    r->lanesPerPool = lanes_per_pool;
    r->F = frames_per_chunk;
    r->elem = encoding == 0 ? 2 : 1;
    const uint32_t lanes = num_zmw / kLane;
    r->pools = (lanes + lanes_per_pool - 1) / lanes_per_pool;
    for (int b = 0; b < 2; ++b)
    {
        const cudaError_t e = cudaEventCreateWithFlags(&r->ev[b], cudaEventDisableTiming);
        if (e != cudaSuccess)
        {
            delete r;
            return Fail(HW_ERR_CUDA, std::string("hw_repacker_create: ") + cudaGetErrorString(e));
        }
    }
    *out = r;
    return HW_OK;
}

int hw_repacker_destroy(hw_repacker* r)
{
    delete r;
    return HW_OK;
}

int hw_repacker_num_pools(const hw_repacker* r, uint32_t* n_pools)
{
    if (!r || !n_pools) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    *n_pools = r->pools;
    return HW_OK;
}

int hw_repack_chunk(hw_repacker* r, const hw_sensor_packet* packets, uint32_t n_packets, const void* d_packet_data,
                    int32_t chunk_first_frame, void* const* d_pool_chunks, void* stream)
{
    if (!r || (n_packets && (!packets || !d_packet_data)) || !d_pool_chunks)
        return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: bad argument");
    const uint32_t e = r->elem;
    const uint32_t line = 64 / e;                 // ZMWs per cache line
    const uint64_t base = reinterpret_cast<uint64_t>(d_packet_data);
    auto& segs = r->host;
    segs.clear();
    for (uint32_t i = 0; i < n_packets; ++i)
    {
        const hw_sensor_packet& p = packets[i];
        const uint32_t W = p.block_width, N = p.num_frames;
        if (W == 0 || W % line != 0)
            return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: block width must be a multiple of the cache-line ZMWs");
        if (p.data_offset % 16 != 0) return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: packet data must be 16-byte aligned");
        if (p.start_frame < chunk_first_frame || (int64_t)p.start_frame + N > (int64_t)chunk_first_frame + r->F)
            return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: packet frames outside the chunk");
        if ((uint64_t)p.start_zmw + (uint64_t)W * p.num_blocks > r->numZmw)
            return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: packet ZMWs outside the chip");
        if (p.start_zmw % line != 0)
            return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: packet start must be cache-line aligned");
        const uint32_t frame0 = (uint32_t)(p.start_frame - chunk_first_frame);
        for (uint32_t b = 0; b < p.num_blocks; ++b)
        {
            const uint32_t zb = p.start_zmw + b * W;
            const uint64_t blockAddr = base + p.data_offset + (uint64_t)b * N * W * e;
            for (uint32_t z0 = zb; z0 < zb + W;)
            {
                const uint32_t lane = z0 / kLane;
                const uint32_t z1 = std::min(zb + W, (lane + 1) * kLane);
                const uint32_t pool = lane / r->lanesPerPool, lip = lane % r->lanesPerPool;
                if (!d_pool_chunks[pool]) return Fail(HW_ERR_INVALID_ARG, "hw_repack_chunk: NULL pool chunk");
                const uint32_t bytes = (z1 - z0) * e;   // 64 or 128
                RepackSeg s;
                s.src = blockAddr + (uint64_t)(z0 - zb) * e;
                s.dst = reinterpret_cast<uint64_t>(d_pool_chunks[pool]) +
                        ((uint64_t)lip * r->F * kLane + (uint64_t)frame0 * kLane + (z0 - lane * kLane)) * e;
                s.rows = N;
                s.vecsLog2 = bytes == 128 ? 3 : 2;
                s.srcStride = W * e;
                s.dstStride = kLane * e;
                segs.push_back(s);
                z0 = z1;
            }
        }
    }
    if (segs.empty()) return HW_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int b = (int)(r->calls & 1);
    // the call that last used staging buffer b must have copied it already
    if (r->inFlight[b] && cudaEventSynchronize(r->ev[b]) != cudaSuccess)
        return Fail(HW_ERR_CUDA, "hw_repack_chunk: event");
    const size_t bytes = segs.size() * sizeof(RepackSeg);
    if (r->stagingCap[b] < bytes)
    {
        cudaFreeHost(r->staging[b]);
        r->staging[b] = nullptr;
        r->stagingCap[b] = 0;
        if (cudaMallocHost((void**)&r->staging[b], bytes) != cudaSuccess)
            return Fail(HW_ERR_CUDA, "hw_repack_chunk: pinned staging");
        r->stagingCap[b] = bytes;
    }
    if (r->devCap < bytes)
    {
        // the previous kernels may still read the old table
        if (cudaStreamSynchronize(s) != cudaSuccess) return Fail(HW_ERR_CUDA, "hw_repack_chunk: sync");
        cudaFree(r->dev);
        r->dev = nullptr;
        r->devCap = 0;
        if (cudaMalloc((void**)&r->dev, bytes) != cudaSuccess) return Fail(HW_ERR_CUDA, "hw_repack_chunk: table");
        r->devCap = bytes;
    }
    std::copy(segs.begin(), segs.end(), r->staging[b]);
    cudaError_t ce = cudaMemcpyAsync(r->dev, r->staging[b], bytes, cudaMemcpyHostToDevice, s);
    if (ce == cudaSuccess) ce = cudaEventRecord(r->ev[b], s);
    if (ce != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_repack_chunk: ") + cudaGetErrorString(ce));
    r->inFlight[b] = true;
    ++r->calls;
    RepackKernel<<<(unsigned)segs.size(), 256, 0, s>>>(r->dev);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_repack_chunk: ") + cudaGetErrorString(ce));
    return HW_OK;
}

}   // extern "C"
