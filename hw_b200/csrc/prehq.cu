// Preliminary HQ stage for sm_100a: PrelimHQFilterBody with its
// BazAggregator packet side (basecaller/appModules/PrelimHQFilter.cpp:63-230,
// bazio/writing/PacketBufferManager.cpp:43-176).
//
// Every chunk's pulses are BAZ-encoded (hw_baz_encoder) into a ring of
// lookback x chunks-per-block slots in device memory, so each ZMW's bytes of
// the last `lookback` metric blocks stay resident.  At a metric block's end
// the stage decides which ZMWs become HQ (the reference's placeholder rule:
// all of them when the preliminary HQ step is off; else, from the
// lookback-th block on, every round(1 / hqThrottleFraction)-th ZMW still
// pre-HQ, in ZMW order -- one exclusive scan; or the caller's marks) and
// writes the block's checkpoint: nothing for a pre-HQ ZMW, its bytes of the
// block for an HQ one, and for a ZMW marked HQ now its bytes of every block
// in the window, oldest first.  Each ZMW's bytes and pulses of each block
// are summed as its chunks arrive, so sizing a checkpoint reads at most
// `lookback` totals a ZMW; a scan places the ZMWs; the copy is a warp per
// ZMW, its pieces (one chunk's bytes of the ZMW each) eight at a time.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "hw_device.cuh"
#include "metric_blocks.cuh"

using namespace hwk;

namespace {

struct Slot
{
    const uint8_t* bytes;
    const uint64_t* offsets;   // [numZmw + 1]
    const uint32_t* events;    // [numZmw]
};

struct RingView
{
    const Slot* slots;         // [lookback][chunksPerBlock]
    const uint32_t* blockBytes;   // [lookback][numZmw] each ZMW's bytes of a block
    const uint32_t* blockEvents;  // [lookback][numZmw]
    uint32_t chunksPerBlock, lookback;
    uint32_t block;            // the metric block ending (count from 0)
    uint32_t chunksInBlock;    // chunks of that block written (a flush may end early)
};

// The slot range of ZMW z's output: HQ before this block -> this block's
// chunks; marked HQ now -> the window's blocks, oldest first.
__device__ __forceinline__ void Window(const RingView& v, bool hq, bool newly, uint32_t& firstBlock, uint32_t& nBlocks)
{
    if (hq)
    {
        firstBlock = v.block;
        nBlocks = 1;
    }
    else if (newly)
    {
        firstBlock = v.block + 1 >= v.lookback ? v.block + 1 - v.lookback : 0;
        nBlocks = v.block + 1 - firstBlock;
    }
    else
    {
        firstBlock = v.block;
        nBlocks = 0;
    }
}

// newly[z]: marked HQ at this block's end.  mode 0: the caller's marks;
// 1: every pre-HQ ZMW; 2: every stride-th pre-HQ ZMW (rank from the scan of
// pre-HQ flags); 3: none.
__global__ void PreFlagKernel(const uint8_t* hq, uint32_t* preHq, uint32_t n)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z < n) preHq[z] = hq[z] ? 0u : 1u;
}

__global__ void MarkKernel(const uint8_t* hq, const uint8_t* marks, const uint32_t* rank, uint32_t stride, int mode,
                           uint8_t* newly, uint32_t n)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= n) return;
    bool m = false;
    if (!hq[z])
    {
        if (mode == 0) m = marks[z] != 0;
        else if (mode == 1) m = true;
        else if (mode == 2) m = rank[z] % stride == 0;
    }
    newly[z] = m ? 1 : 0;
}

// Piece j (0 <= j < pieces) of ZMW z's output: chunk c of block b of the
// window [b0, b0 + nb); the block ending has v.chunksInBlock chunks.
__device__ __forceinline__ const Slot& PieceSlot(const RingView& v, uint32_t b0, uint32_t nb, uint32_t j)
{
    const uint32_t full = (nb - 1) * v.chunksPerBlock;   // pieces of the blocks before the one ending
    const uint32_t b = j < full ? b0 + j / v.chunksPerBlock : v.block;
    const uint32_t c = j < full ? j % v.chunksPerBlock : j - full;
    return v.slots[(size_t)(b % v.lookback) * v.chunksPerBlock + c];
}

__device__ __forceinline__ uint32_t Pieces(const RingView& v, uint32_t nb)
{
    return nb ? (nb - 1) * v.chunksPerBlock + v.chunksInBlock : 0;
}

// Each ZMW's bytes and pulses of the block so far, after each chunk.
__global__ void BlockTotalsKernel(const uint64_t* offsets, const uint32_t* events, bool first, uint32_t* bytes,
                                  uint32_t* evs, uint32_t n)
{
    for (uint32_t z = blockIdx.x * blockDim.x + threadIdx.x; z < n; z += gridDim.x * blockDim.x)
    {
        const uint32_t b = (uint32_t)(offsets[z + 1] - offsets[z]), e = events[z];
        bytes[z] = first ? b : bytes[z] + b;
        evs[z] = first ? e : evs[z] + e;
    }
}

// offsets[z] = the checkpoint bytes of ZMW z (scanned afterwards; offsets[n]
// = 0 becomes the total), events[z] its pulses: from the block totals.
__global__ void CheckpointSizeKernel(RingView v, const uint8_t* hq, const uint8_t* newly, bool flush,
                                     uint64_t* offsets, uint32_t* events, uint32_t n)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) offsets[n] = 0;
    for (uint32_t z = blockIdx.x * blockDim.x + threadIdx.x; z < n; z += gridDim.x * blockDim.x)
    {
        uint32_t b0, nb;
        Window(v, hq[z] != 0, !flush && newly[z] != 0, b0, nb);
        if (v.chunksInBlock == 0 && nb) --nb;   // a flush right after a block's end: nothing written yet
        uint64_t bytes = 0;
        uint32_t ev = 0;
        for (uint32_t b = b0; b < b0 + nb; ++b)
        {
            const size_t at = (size_t)(b % v.lookback) * n + z;
            bytes += v.blockBytes[at];
            ev += v.blockEvents[at];
        }
        offsets[z] = bytes;
        events[z] = ev;
    }
}

constexpr int kCopyBatch = 8;   // pieces whose first 32 bytes a warp loads at once

// A warp per 32 ZMWs (grid-stride): each lane reads one ZMW's window and
// place (coalesced), a ballot skips the ZMWs with nothing to copy, and for
// each of the others the lanes read up to 32 pieces' places at once and copy
// the pieces eight at a time, each across the warp (coalesced bytes, the
// eight loads in flight together).
__global__ void __launch_bounds__(256) CheckpointCopyKernel(RingView v, const uint8_t* hq, const uint8_t* newly,
                                                            bool flush, const uint64_t* offsets, uint8_t* out,
                                                            uint32_t n)
{
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warps = gridDim.x * (blockDim.x / 32);
    for (uint32_t zb = (blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32) * 32; zb < n; zb += warps * 32)
    {
        const uint32_t zl = zb + lane;
        uint32_t myB0 = 0, myNb = 0;
        uint64_t myDst = 0;
        if (zl < n)
        {
            Window(v, hq[zl] != 0, !flush && newly[zl] != 0, myB0, myNb);
            myDst = offsets[zl];
            if (offsets[zl + 1] == myDst) myNb = 0;   // nothing to copy
        }
        uint32_t busy = __ballot_sync(~0u, myNb != 0);
        while (busy)
        {
            const uint32_t who = __ffs(busy) - 1;
            busy &= busy - 1;
            const uint32_t z = zb + who;
            const uint32_t b0 = __shfl_sync(~0u, myB0, who), nb = __shfl_sync(~0u, myNb, who);
            uint8_t* dst = out + __shfl_sync(~0u, myDst, who);
            const uint32_t pieces = Pieces(v, nb);
            for (uint32_t j0 = 0; j0 < pieces; j0 += 32)
            {
                const uint32_t j = j0 + lane;
                const uint8_t* src = nullptr;
                uint32_t len = 0;
                if (j < pieces)
                {
                    const Slot& sl = PieceSlot(v, b0, nb, j);
                    const uint64_t lo = sl.offsets[z];
                    len = (uint32_t)(sl.offsets[z + 1] - lo);
                    src = sl.bytes + lo;
                }
                uint32_t incl = len;   // each piece's place: a warp scan of the lengths
#pragma unroll
                for (int o = 1; o < 32; o <<= 1)
                {
                    const uint32_t t = __shfl_up_sync(~0u, incl, o);
                    if (lane >= (uint32_t)o) incl += t;
                }
                const uint32_t excl = incl - len;
                const uint32_t m = min(32u, pieces - j0);
                for (uint32_t q0 = 0; q0 < m; q0 += kCopyBatch)
                {
                    const uint8_t* ps[kCopyBatch];
                    uint32_t pl[kCopyBatch], po[kCopyBatch];
                    uint8_t x[kCopyBatch];
#pragma unroll
                    for (int k = 0; k < kCopyBatch; ++k)
                    {
                        const uint32_t q = (q0 + k) & 31;
                        ps[k] = reinterpret_cast<const uint8_t*>(
                            __shfl_sync(~0u, reinterpret_cast<uintptr_t>(src), q));
                        pl[k] = __shfl_sync(~0u, len, q);
                        po[k] = __shfl_sync(~0u, excl, q);
                        if (q0 + k >= m) pl[k] = 0;
                        x[k] = lane < pl[k] ? ps[k][lane] : 0;
                    }
#pragma unroll
                    for (int k = 0; k < kCopyBatch; ++k)
                    {
                        if (lane < pl[k]) dst[po[k] + lane] = x[k];
                        for (uint32_t i = 32 + lane; i < pl[k]; i += 32) dst[po[k] + i] = ps[k][i];
                    }
                }
                dst += __shfl_sync(~0u, incl, 31);
            }
        }
    }
}

__global__ void PromoteKernel(uint8_t* hq, const uint8_t* newly, uint32_t n, unsigned long long* count)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    bool m = false;
    if (z < n && newly[z])
    {
        hq[z] = 1;
        m = true;
    }
    const uint32_t votes = __popc(__ballot_sync(~0u, m));
    if ((threadIdx.x & 31) == 0 && votes) atomicAdd(count, (unsigned long long)votes);
}

// The most recent activity label of each ZMW the aggregator is given
// metrics for (z % stride == 0, PrelimHQFilter.cpp:107-118) from a block's
// HF metrics.
__global__ void ActivityKernel(const hw_basecalling_metrics* metrics, uint8_t* activity, uint32_t n, uint32_t stride)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z < n && z % stride == 0) activity[z] = metrics[z / kLane].activity_label[z % kLane];
}

int Fail(int code, const std::string& msg) { return hwk::SetLastError(code, msg.c_str()); }

int Cuda(cudaError_t e, const char* where)
{
    return e == cudaSuccess ? HW_OK : Fail(HW_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

}   // namespace

struct hw_prelim_hq
{
    hw_prelim_hq_config cfg{};
    uint32_t numZmw = 0, stride = 1;
    hw_baz_encoder* enc = nullptr;
    struct HostSlot
    {
        uint8_t* bytes = nullptr;
        uint64_t cap = 0;
        uint64_t* offsets = nullptr;
        uint32_t* events = nullptr;
    };
    std::vector<HostSlot> slots;       // [lookback][chunksPerBlock]
    Slot* dSlots = nullptr;            // device copy of the slot table
    uint32_t block = 0, chunk = 0;     // blocks ended; chunks of the current block written
    uint64_t seen = 0;                 // blocks the placeholder rule has seen
    uint8_t* hq = nullptr;             // [numZmw]
    uint8_t* newly = nullptr;          // [numZmw]
    uint32_t* rank = nullptr;          // [numZmw + 1]
    uint32_t* blockBytes = nullptr;    // [lookback][numZmw]
    uint32_t* blockEvents = nullptr;   // [lookback][numZmw]
    uint8_t* activity = nullptr;       // [numZmw]
    uint8_t* out = nullptr;            // checkpoint bytes
    uint64_t outCap = 0;
    uint64_t* outOffsets = nullptr;    // [numZmw + 1]
    uint32_t* outEvents = nullptr;     // [numZmw]
    unsigned long long* numHq = nullptr;
    void* scanTmp = nullptr;
    size_t scanBytes = 0;
    // metric side (cfg.metrics)
    MetricSide ms{};
    hw_spider_metric_block* mOut = nullptr;
    uint64_t mCap = 0, mTotal = 0;
    uint64_t* mOffsets = nullptr;      // [numZmw + 1]
    uint32_t mBlock = 0;

    ~hw_prelim_hq()
    {
        cudaDeviceSynchronize();
        hw_baz_encoder_destroy(enc);
        for (auto& s : slots)
        {
            cudaFree(s.bytes);
            cudaFree(s.offsets);
            cudaFree(s.events);
        }
        cudaFree(dSlots);
        cudaFree(hq);
        cudaFree(newly);
        cudaFree(rank);
        cudaFree(blockBytes);
        cudaFree(blockEvents);
        cudaFree(activity);
        cudaFree(out);
        cudaFree(outOffsets);
        cudaFree(outEvents);
        cudaFree(numHq);
        cudaFree(scanTmp);
        cudaFree(ms.ring);
        cudaFree(ms.agg);
        cudaFree(ms.pending);
        cudaFree(ms.pendingCount);
        cudaFree(mOut);
        cudaFree(mOffsets);
    }

    // The metric side of the checkpoint: before the promotion of the ZMWs
    // marked now (hq = HQ before this block's end).
    int MetricCheckpoint(bool flush, cudaStream_t s)
    {
        const uint32_t n = numZmw, threads = 256, blocks = (n + threads - 1) / threads;
        const int mode = flush ? 1 : 0;
        MetricCountKernel<<<blocks, threads, 0, s>>>(ms, hq, newly, block, mode, mOffsets);
        int rc = Cuda(cudaGetLastError(), "hw_prelim_hq metrics");
        if (!rc)
            rc = Cuda(cub::DeviceScan::ExclusiveSum(scanTmp, scanBytes, mOffsets, mOffsets, (int)n + 1, s),
                      "hw_prelim_hq metrics");
        uint64_t total = 0;
        if (!rc) rc = Cuda(cudaMemcpyAsync(&total, mOffsets + n, sizeof(total), cudaMemcpyDeviceToHost, s),
                           "hw_prelim_hq metrics");
        if (!rc) rc = Cuda(cudaStreamSynchronize(s), "hw_prelim_hq metrics");
        if (rc) return rc;
        if (total > mCap)
        {
            cudaFree(mOut);
            mOut = nullptr;
            mCap = 0;
            const uint64_t cap = std::max<uint64_t>(total + total / 4, 1024);
            if ((rc = Cuda(cudaMalloc((void**)&mOut, cap * sizeof(hw_spider_metric_block)), "hw_prelim_hq metrics")))
                return rc;
            mCap = cap;
        }
        MetricWriteKernel<<<blocks, threads, 0, s>>>(ms, hq, newly, block, mode, mOffsets, mOut);
        if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq metrics"))) return rc;
        mTotal = total;
        mBlock = block;
        return HW_OK;
    }

    int UploadSlots()
    {
        std::vector<Slot> t(slots.size());
        for (size_t i = 0; i < slots.size(); ++i) t[i] = Slot{slots[i].bytes, slots[i].offsets, slots[i].events};
        return Cuda(cudaMemcpy(dSlots, t.data(), sizeof(Slot) * t.size(), cudaMemcpyHostToDevice), "hw_prelim_hq");
    }

    // The checkpoint of the block ending now (flush: the chunks so far, no marking).
    int Checkpoint(const uint8_t* marks, bool flush, hw_baz_checkpoint* res, cudaStream_t s)
    {
        const uint32_t n = numZmw, threads = 256, blocks = (n + threads - 1) / threads;
        int rc;
        if (!flush)
        {
            int mode;
            if (marks) mode = 0, ++seen;
            else if (!cfg.enable_prehq) mode = 1;
            else mode = ++seen < cfg.lookback_blocks ? 3 : 2;
            if (mode == 2)
            {
                PreFlagKernel<<<blocks, threads, 0, s>>>(hq, rank, n);
                if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq"))) return rc;
                if ((rc = Cuda(cub::DeviceScan::ExclusiveSum(scanTmp, scanBytes, rank, rank, (int)n, s),
                               "hw_prelim_hq")))
                    return rc;
            }
            MarkKernel<<<blocks, threads, 0, s>>>(hq, marks, rank, stride, mode, newly, n);
            if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq"))) return rc;
        }
        const RingView v{dSlots, blockBytes, blockEvents, cfg.chunks_per_block, cfg.lookback_blocks, block,
                         flush ? chunk : cfg.chunks_per_block};
        const uint32_t grid = std::min<uint32_t>(blocks, 148 * 16);
        CheckpointSizeKernel<<<grid, threads, 0, s>>>(v, hq, newly, flush, outOffsets, outEvents, n);
        if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq"))) return rc;
        if ((rc = Cuda(cub::DeviceScan::ExclusiveSum(scanTmp, scanBytes, outOffsets, outOffsets, (int)n + 1, s),
                       "hw_prelim_hq")))
            return rc;
        uint64_t total = 0;
        if ((rc = Cuda(cudaMemcpyAsync(&total, outOffsets + n, sizeof(total), cudaMemcpyDeviceToHost, s),
                       "hw_prelim_hq")))
            return rc;
        if ((rc = Cuda(cudaStreamSynchronize(s), "hw_prelim_hq"))) return rc;
        if (total > outCap)
        {
            cudaFree(out);
            out = nullptr;
            outCap = 0;
            const uint64_t cap = std::max<uint64_t>(total + total / 4, 1 << 20);
            if ((rc = Cuda(cudaMalloc((void**)&out, cap), "hw_prelim_hq"))) return rc;
            outCap = cap;
        }
        CheckpointCopyKernel<<<std::min<uint32_t>((n + 255) / 256, 148 * 8), 256, 0, s>>>(v, hq, newly, flush,
                                                                                           outOffsets, out, n);
        if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq"))) return rc;
        if (cfg.metrics && (rc = MetricCheckpoint(flush, s))) return rc;
        if (!flush)
        {
            PromoteKernel<<<blocks, threads, 0, s>>>(hq, newly, n, numHq);
            if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq"))) return rc;
        }
        unsigned long long nHq = 0;
        if ((rc = Cuda(cudaMemcpyAsync(&nHq, numHq, sizeof(nHq), cudaMemcpyDeviceToHost, s), "hw_prelim_hq")))
            return rc;
        if ((rc = Cuda(cudaStreamSynchronize(s), "hw_prelim_hq"))) return rc;
        res->d_bytes = out;
        res->total_bytes = total;
        res->d_offsets = outOffsets;
        res->d_events = outEvents;
        res->d_hq = hq;
        res->num_hq = (uint32_t)nHq;
        res->block = block;
        return HW_OK;
    }
};

extern "C" {

int hw_prelim_hq_config_default(hw_prelim_hq_config* cfg)
{
    if (!cfg) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    *cfg = hw_prelim_hq_config{};
    cfg->chunks_per_block = 8;          // framesPerHFMetricBlock 4096 / 512-frame chunks
    cfg->lookback_blocks = 10;          // PrelimHQConfig lookbackSize
    cfg->enable_prehq = 0;              // enablePreHQ
    cfg->hq_throttle_fraction = 0.10f;  // hqThrottleFraction
    cfg->zmw_stride = 1;                // zmwOutputStride
    return HW_OK;
}

int hw_prelim_hq_create(const hw_baz_field* fields, uint32_t n_fields, int32_t skip_rejects, uint32_t num_zmw,
                        const hw_prelim_hq_config* cfg, hw_prelim_hq** out)
{
    if (!out || !cfg || num_zmw == 0 || cfg->chunks_per_block == 0 || cfg->lookback_blocks == 0 ||
        !(cfg->hq_throttle_fraction > 0.f) || cfg->zmw_stride == 0 || 64 % cfg->zmw_stride != 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_prelim_hq_create: bad argument");
    *out = nullptr;
    auto h = new hw_prelim_hq;
    h->cfg = *cfg;
    h->numZmw = num_zmw;
    // DummyPreHQ: stride = round(1 / hqThrottleFraction)
    h->stride = (uint32_t)std::max(1.0f, std::round(1 / cfg->hq_throttle_fraction));
    int rc = hw_baz_encoder_create(fields, n_fields, skip_rejects, num_zmw, &h->enc);
    if (!rc) rc = hw_baz_encoder_set_zmw_stride(h->enc, cfg->zmw_stride);
    h->slots.resize((size_t)cfg->lookback_blocks * cfg->chunks_per_block);
    for (auto& s : h->slots)
    {
        if (rc) break;
        s.cap = (uint64_t)num_zmw * 32;   // grows when a chunk needs more
        rc = Cuda(cudaMalloc((void**)&s.bytes, s.cap), "hw_prelim_hq_create");
        if (!rc) rc = Cuda(cudaMalloc((void**)&s.offsets, sizeof(uint64_t) * (num_zmw + 1)), "hw_prelim_hq_create");
        if (!rc) rc = Cuda(cudaMemset(s.offsets, 0, sizeof(uint64_t) * (num_zmw + 1)), "hw_prelim_hq_create");
        if (!rc) rc = Cuda(cudaMalloc((void**)&s.events, sizeof(uint32_t) * num_zmw), "hw_prelim_hq_create");
        if (!rc) rc = Cuda(cudaMemset(s.events, 0, sizeof(uint32_t) * num_zmw), "hw_prelim_hq_create");
    }
    auto alloc = [&](void** p, size_t bytes) {
        if (!rc) rc = Cuda(cudaMalloc(p, bytes), "hw_prelim_hq_create");
        if (!rc) rc = Cuda(cudaMemset(*p, 0, bytes), "hw_prelim_hq_create");
    };
    alloc((void**)&h->dSlots, sizeof(Slot) * h->slots.size());
    alloc((void**)&h->hq, num_zmw);
    alloc((void**)&h->newly, num_zmw);
    alloc((void**)&h->rank, sizeof(uint32_t) * (num_zmw + 1));
    alloc((void**)&h->blockBytes, sizeof(uint32_t) * (size_t)cfg->lookback_blocks * num_zmw);
    alloc((void**)&h->blockEvents, sizeof(uint32_t) * (size_t)cfg->lookback_blocks * num_zmw);
    alloc((void**)&h->activity, num_zmw);
    alloc((void**)&h->outOffsets, sizeof(uint64_t) * (num_zmw + 1));
    alloc((void**)&h->outEvents, sizeof(uint32_t) * num_zmw);
    alloc((void**)&h->numHq, sizeof(unsigned long long));
    if (!rc) rc = Cuda(cudaMemset(h->activity, 4, num_zmw), "hw_prelim_hq_create");   // NUM_PHYS_STATES: none yet
    if (cfg->metrics)
    {
        MetricSide& m = h->ms;
        m.numZmw = num_zmw;
        m.lookback = cfg->lookback_blocks;
        m.stride = cfg->zmw_stride;
        m.production = cfg->enable_prehq != 0;
        if (m.production)
        {
            alloc((void**)&m.ring, sizeof(MetricBlk) * (size_t)cfg->lookback_blocks * num_zmw);
            alloc((void**)&m.agg, sizeof(AggBlk) * (size_t)num_zmw);
        }
        alloc((void**)&m.pending, sizeof(hw_spider_metric_block) * (size_t)num_zmw);
        alloc((void**)&m.pendingCount, num_zmw);
        alloc((void**)&h->mOffsets, sizeof(uint64_t) * (num_zmw + 1));
        if (!rc)
        {
            MetricInitKernel<<<(num_zmw + 255) / 256, 256>>>(m);
            rc = Cuda(cudaGetLastError(), "hw_prelim_hq_create");
            if (!rc) rc = Cuda(cudaStreamSynchronize(0), "hw_prelim_hq_create");
        }
    }
    if (!rc)
    {
        size_t a = 0, b = 0;
        rc = Cuda(cub::DeviceScan::ExclusiveSum(nullptr, a, h->outOffsets, h->outOffsets, (int)num_zmw + 1),
                  "hw_prelim_hq_create");
        if (!rc) rc = Cuda(cub::DeviceScan::ExclusiveSum(nullptr, b, h->rank, h->rank, (int)num_zmw), "hw_prelim_hq_create");
        h->scanBytes = std::max(a, b);
        if (!rc) rc = Cuda(cudaMalloc(&h->scanTmp, h->scanBytes), "hw_prelim_hq_create");
    }
    if (!rc) rc = h->UploadSlots();
    if (rc)
    {
        delete h;
        return rc;
    }
    *out = h;
    return HW_OK;
}

int hw_prelim_hq_destroy(hw_prelim_hq* h)
{
    delete h;
    return HW_OK;
}

int hw_prelim_hq_process(hw_prelim_hq* h, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                         const hw_basecalling_metrics* d_metrics, const uint8_t* d_marks, int32_t* produced,
                         hw_baz_checkpoint* out, void* stream)
{
    const NvtxRange range("hw_prelim_hq_process");
    if (!h || !d_pulses || !d_lens || !produced || !out || max_calls == 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_prelim_hq_process: bad argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    *produced = 0;
    const uint32_t n = h->numZmw;
    auto& slot = h->slots[(size_t)(h->block % h->cfg.lookback_blocks) * h->cfg.chunks_per_block + h->chunk];
    // the slot held the chunk of `lookback` blocks ago, out of the window now
    uint64_t total = 0;
    int rc = hw_baz_encode(h->enc, d_pulses, d_lens, max_calls, slot.bytes, slot.cap, slot.offsets, slot.events,
                           &total, stream);
    if (rc == HW_ERR_OUT_OF_MEMORY)
    {
        cudaFree(slot.bytes);   // waits for the device: nothing reads the old slot afterwards
        slot.bytes = nullptr;
        slot.cap = 0;
        const uint64_t cap = total + total / 4 + 64;
        if ((rc = Cuda(cudaMalloc((void**)&slot.bytes, cap), "hw_prelim_hq_process"))) return rc;
        slot.cap = cap;
        if ((rc = h->UploadSlots())) return rc;
        rc = hw_baz_encode(h->enc, d_pulses, d_lens, max_calls, slot.bytes, slot.cap, slot.offsets, slot.events,
                           &total, stream);
    }
    if (rc) return rc;
    const uint32_t threads = 256, blocks = (n + threads - 1) / threads;
    const size_t at = (size_t)(h->block % h->cfg.lookback_blocks) * n;
    BlockTotalsKernel<<<std::min<uint32_t>(blocks, 148 * 16), threads, 0, s>>>(
        slot.offsets, slot.events, h->chunk == 0, h->blockBytes + at, h->blockEvents + at, n);
    if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq_process"))) return rc;
    if (d_metrics)
    {
        ActivityKernel<<<blocks, threads, 0, s>>>(d_metrics, h->activity, n, h->cfg.zmw_stride);
        if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq_process"))) return rc;
        if (h->cfg.metrics)
        {
            MetricAddKernel<<<blocks, threads, 0, s>>>(h->ms, d_metrics, h->hq, h->block);
            if ((rc = Cuda(cudaGetLastError(), "hw_prelim_hq_process"))) return rc;
        }
    }
    if (++h->chunk < h->cfg.chunks_per_block) return HW_OK;
    rc = h->Checkpoint(d_marks, false, out, s);
    if (rc) return rc;
    *produced = 1;
    h->chunk = 0;
    ++h->block;
    return HW_OK;
}

int hw_prelim_hq_flush(hw_prelim_hq* h, int32_t* produced, hw_baz_checkpoint* out, void* stream)
{
    if (!h || !produced || !out) return Fail(HW_ERR_INVALID_ARG, "hw_prelim_hq_flush: bad argument");
    *produced = 0;
    const int rc = h->Checkpoint(nullptr, true, out, reinterpret_cast<cudaStream_t>(stream));
    if (rc) return rc;
    *produced = 1;
    return HW_OK;
}

int hw_prelim_hq_metrics(const hw_prelim_hq* h, hw_metric_checkpoint* out)
{
    if (!h || !out) return Fail(HW_ERR_INVALID_ARG, "hw_prelim_hq_metrics: bad argument");
    if (!h->cfg.metrics) return Fail(HW_ERR_INVALID_ARG, "hw_prelim_hq_metrics: the stage runs no metric side");
    *out = hw_metric_checkpoint{};
    out->d_blocks = h->mOut;
    out->total_blocks = h->mTotal;
    out->d_offsets = h->mOffsets;
    out->block = h->mBlock;
    return HW_OK;
}

int hw_prelim_hq_activity(hw_prelim_hq* h, uint8_t* d_out, void* stream)
{
    if (!h || !d_out) return Fail(HW_ERR_INVALID_ARG, "hw_prelim_hq_activity: bad argument");
    return Cuda(cudaMemcpyAsync(d_out, h->activity, h->numZmw, cudaMemcpyDeviceToDevice,
                                reinterpret_cast<cudaStream_t>(stream)),
                "hw_prelim_hq_activity");
}

}   // extern "C"
