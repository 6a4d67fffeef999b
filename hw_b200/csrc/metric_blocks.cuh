// Metric side of the preliminary HQ stage for sm_100a: the BazAggregator's
// MetricBufferManager (bazio/writing/MetricBufferManager.h:70-357) over the
// reference's metric-block types (basecaller/dataTypes/Metrics.h:36-366).
//
// Every ZMW is independent, so each kernel is a thread per ZMW:
//  - MetricAddKernel (a block's HF metrics arrive): with the preliminary HQ
//    step off, CompleteMetrics<uint16_t, half> converted straight into the
//    ZMW's pending output; on, a pre-HQ ZMW's ProductionMetrics<uint16_t,
//    half> goes into its slot of the lookback ring, an HQ ZMW's is
//    aggregated into its open aggregate (ProductionMetrics<uint32_t,
//    float>), which is emitted first when the activity label changes
//    (AddProductionMetrics, :252-287);
//  - at a block's end, MetricCountKernel sizes each ZMW's output (its
//    pending block, or for a ZMW marked HQ now the label runs of its window,
//    NumTransitionsInLookbackWindow :289-305), a scan places them, and
//    MetricWriteKernel writes them: pending blocks; for a newly-HQ ZMW its
//    pre-HQ aggregate and the window's runs but the last, which becomes its
//    open aggregate (UpdateLookback :180-233, AddLookbackWindowMetricBlocks
//    :307-333); a ZMW staying pre-HQ aggregates its oldest ring slot into
//    its pre-HQ aggregate once the window is full and clears the slot for
//    the next block;
//  - the flush emits every open aggregate with data (Flush :161-178).
// Each ZMW follows its own entries and aggregate; the reference's two index
// slips (an HQ ZMW's aggregate looked up at a stale window index, :263, and
// the window walk reading each buffer at the index of the buffer before it,
// :318) are not reproduced -- they read other ZMWs' data, or memory never
// written, once ZMWs below were marked HQ inside the window.
//
// Arithmetic follows Metrics.h:73-146 exactly: every product, sum and
// quotient a separately rounded float operation (no contraction), counts
// converted to float, float -> half round-to-nearest-even
// (__float2half_rn), half sqrt as the half rounding of the float sqrt.
#pragma once

#include <cuda_fp16.h>

#include "hw_device.cuh"

namespace hwk {

constexpr uint8_t kNoActivity = 4;   // HQRFPhysicalStates::NUM_PHYS_STATES

// ProductionMetrics<uint16_t, half_float::half> (48 bytes; halves as bits).
struct __align__(16) MetricBlk
{
    uint16_t numFrames, pulseWidth, baseWidth, numPulses, numBases, numBaselineFrames;
    uint16_t pkmid[4];
    uint16_t numPkmidFrames[4];
    uint16_t numBasesByAnalog[4];
    uint16_t var, mean;
    uint8_t label, pad0;
    uint16_t pad1[3];
};
static_assert(sizeof(MetricBlk) == 48, "MetricBlk");

// ProductionMetrics<uint32_t, float> (the aggregate).
struct __align__(16) AggBlk
{
    uint32_t numFrames, pulseWidth, baseWidth, numPulses, numBases, numBaselineFrames;
    float pkmid[4];
    uint32_t numPkmidFrames[4];
    uint32_t numBasesByAnalog[4];
    float var, mean;
    uint32_t label;
    uint32_t pad;
};
static_assert(sizeof(AggBlk) == 96, "AggBlk");

__device__ __forceinline__ uint16_t ToHalf(float x) { return __half_as_ushort(__float2half_rn(x)); }
__device__ __forceinline__ float FromHalf(uint16_t h) { return __half2float(__ushort_as_half(h)); }
__device__ __forceinline__ float U2F(uint32_t v) { return __uint2float_rn(v); }

__device__ __forceinline__ MetricBlk EmptyMetricBlk()
{
    MetricBlk m = {};
    m.label = kNoActivity;
    return m;
}

__device__ __forceinline__ AggBlk EmptyAggBlk()
{
    AggBlk a = {};
    a.label = kNoActivity;
    return a;
}

// ProductionMetrics(bm, z), Metrics.h:53-70
__device__ __forceinline__ MetricBlk MetricFromHf(const hw_basecalling_metrics& bm, int z)
{
    MetricBlk m = {};
    m.numFrames = bm.num_frames[z];
    m.pulseWidth = bm.num_pulse_frames[z];
    m.baseWidth = bm.num_base_frames[z];
    m.numPulses = bm.num_pulses[z];
    m.numBases = bm.num_bases[z];
    m.numBaselineFrames = bm.num_frames_baseline[z];
    m.var = ToHalf(bm.frame_baseline_variance_dws[z]);
    m.mean = ToHalf(bm.frame_baseline_dws[z]);
    m.label = bm.activity_label[z];
#pragma unroll
    for (int a = 0; a < 4; ++a)
    {
        const uint16_t n = bm.num_pk_mid_frames[a][z];
        m.numPkmidFrames[a] = n;
        m.pkmid[a] = ToHalf(n > 0 ? __fdiv_rn(bm.pk_mid_signal[a][z], U2F(n)) : 0.0f);
        m.numBasesByAnalog[a] = bm.num_bases_by_analog[a][z];
    }
    return m;
}

// The uint16/half block with its values widened (exact), for Aggregate.
__device__ __forceinline__ AggBlk Widen(const MetricBlk& m)
{
    AggBlk w;
    w.numFrames = m.numFrames;
    w.pulseWidth = m.pulseWidth;
    w.baseWidth = m.baseWidth;
    w.numPulses = m.numPulses;
    w.numBases = m.numBases;
    w.numBaselineFrames = m.numBaselineFrames;
#pragma unroll
    for (int a = 0; a < 4; ++a)
    {
        w.pkmid[a] = FromHalf(m.pkmid[a]);
        w.numPkmidFrames[a] = m.numPkmidFrames[a];
        w.numBasesByAnalog[a] = m.numBasesByAnalog[a];
    }
    w.var = FromHalf(m.var);
    w.mean = FromHalf(m.mean);
    w.label = m.label;
    w.pad = 0;
    return w;
}

// ProductionMetrics<uint32_t, float>::Aggregate, Metrics.h:73-118
__device__ __forceinline__ void AggAdd(AggBlk& a, const AggBlk& b)
{
    const uint32_t nbf = a.numBaselineFrames + b.numBaselineFrames;
    float mean = __fadd_rn(__fmul_rn(U2F(a.numBaselineFrames), a.mean), __fmul_rn(U2F(b.numBaselineFrames), b.mean));
    if (nbf > 0)
    {
        mean = __fdiv_rn(mean, U2F(nbf));
        float bv = 0.0f;
        uint32_t nk = nbf;
        const uint32_t n0 = a.numBaselineFrames > 1 ? a.numBaselineFrames - 1 : a.numBaselineFrames;
        bv = __fadd_rn(bv, __fmul_rn(U2F(n0), a.var));
        if (a.numBaselineFrames > 0) --nk;
        const uint32_t n1 = b.numBaselineFrames > 1 ? b.numBaselineFrames - 1 : b.numBaselineFrames;
        bv = __fadd_rn(bv, __fmul_rn(U2F(n1), b.var));
        if (b.numBaselineFrames > 0) --nk;
        a.var = __fdiv_rn(bv, U2F(nk));
        a.numBaselineFrames = nbf;
    }
    a.mean = mean;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        float p = __fadd_rn(__fmul_rn(U2F(a.numPkmidFrames[k]), a.pkmid[k]), __fmul_rn(U2F(b.numPkmidFrames[k]), b.pkmid[k]));
        a.numPkmidFrames[k] += b.numPkmidFrames[k];
        if (a.numPkmidFrames[k] > 0) p = __fdiv_rn(p, U2F(a.numPkmidFrames[k]));
        a.pkmid[k] = p;
        a.numBasesByAnalog[k] += b.numBasesByAnalog[k];
    }
    a.numFrames += b.numFrames;
    a.pulseWidth += b.pulseWidth;
    a.baseWidth += b.baseWidth;
    a.numPulses += b.numPulses;
    a.numBases += b.numBases;
    a.label = b.label;
}

__device__ __forceinline__ void ZeroSpider(hw_spider_metric_block& s)
{
    uint32_t* w = reinterpret_cast<uint32_t*>(&s);
#pragma unroll
    for (int i = 0; i < (int)(sizeof(hw_spider_metric_block) / 4); ++i) w[i] = 0;
}

// ProductionMetrics<uint32_t, float>::Convert, Metrics.h:121-146, through the
// uint16_t setters of bazio/MetricBlock.h:153-310
__device__ __forceinline__ void AggToSpider(const AggBlk& a, hw_spider_metric_block& s)
{
    ZeroSpider(s);
    s.num_frames = (uint16_t)a.numFrames;
    s.pulse_width = (uint16_t)a.pulseWidth;
    s.base_width = (uint16_t)a.baseWidth;
    s.num_pulses = (uint16_t)a.numPulses;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        s.pkmid[k] = a.pkmid[k];
        s.num_pkmid_frames[k] = (uint16_t)a.numPkmidFrames[k];
        s.num_bases[k] = (uint16_t)a.numBasesByAnalog[k];
    }
    s.baseline = a.mean;
    s.baseline_sd = __fsqrt_rn(a.var);
    s.num_baseline_frames = a.numBaselineFrames;
    s.activity_label = (uint8_t)a.label;
}

// CompleteMetrics<uint16_t, half>(bm, z) converted, Metrics.h:212-228 and
// :288-318 (with ProductionMetrics<uint16_t, half>::Convert)
__device__ __forceinline__ void CompleteToSpider(const hw_basecalling_metrics& bm, int z, hw_spider_metric_block& s)
{
    const MetricBlk m = MetricFromHf(bm, z);
    ZeroSpider(s);
    s.num_frames = m.numFrames;
    s.pulse_width = m.pulseWidth;
    s.base_width = m.baseWidth;
    s.num_pulses = m.numPulses;
#pragma unroll
    for (int k = 0; k < 4; ++k)
    {
        s.pkmid[k] = FromHalf(m.pkmid[k]);
        s.num_pkmid_frames[k] = m.numPkmidFrames[k];
        s.num_bases[k] = m.numBasesByAnalog[k];
        s.pkmax[k] = FromHalf(ToHalf(bm.pk_max[k][z]));
        s.num_pkmid_bases[k] = bm.num_pk_mid_bases_by_analog[k][z];
        s.bpzvar[k] = FromHalf(ToHalf(bm.bp_zvar[k][z]));
        s.pkzvar[k] = FromHalf(ToHalf(bm.pk_zvar[k][z]));
    }
    s.baseline = FromHalf(m.mean);
    s.baseline_sd = FromHalf(ToHalf(__fsqrt_rn(FromHalf(m.var))));   // half sqrt
    s.num_baseline_frames = m.numBaselineFrames;
    s.activity_label = m.label;
    s.num_half_sandwiches = bm.num_half_sandwiches[z];
    s.num_sandwiches = bm.num_sandwiches[z];
    s.num_pulse_label_stutters = bm.num_pulse_label_stutters[z];
    s.pulse_detection_score = FromHalf(ToHalf(bm.pulse_detection_score[z]));
    s.trace_autocorr = FromHalf(ToHalf(bm.autocorrelation[z]));
}

struct MetricSide
{
    MetricBlk* ring;                 // [lookback][numZmw] (preliminary HQ on)
    AggBlk* agg;                     // [numZmw] open aggregates
    hw_spider_metric_block* pending; // [numZmw]
    uint8_t* pendingCount;           // [numZmw] 0 or 1
    uint32_t numZmw, lookback, stride;
    int production;
};

__global__ void MetricInitKernel(MetricSide S)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= S.numZmw) return;
    S.pendingCount[z] = 0;
    if (!S.production) return;
    S.agg[z] = EmptyAggBlk();
    for (uint32_t w = 0; w < S.lookback; ++w) S.ring[(size_t)w * S.numZmw + z] = EmptyMetricBlk();
}

// AddZmw of every ZMW z with z % stride == 0 (PrelimHQFilter.cpp:107-118,
// MetricBufferManager.h:142-149): hq = HQ before this block's end.
__global__ void MetricAddKernel(MetricSide S, const hw_basecalling_metrics* __restrict__ hf, const uint8_t* hq,
                                uint32_t block)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= S.numZmw || z % S.stride) return;
    const hw_basecalling_metrics& bm = hf[z / kLane];
    const int lz = (int)(z % kLane);
    if (!S.production)
    {
        CompleteToSpider(bm, lz, S.pending[z]);
        S.pendingCount[z] = 1;
        return;
    }
    const MetricBlk m = MetricFromHf(bm, lz);
    if (!hq[z])
    {
        S.ring[(size_t)(block % S.lookback) * S.numZmw + z] = m;
        return;
    }
    AggBlk a = S.agg[z];
    const AggBlk w = Widen(m);
    if (w.label != a.label)
    {
        if (a.label != kNoActivity)
        {
            AggToSpider(a, S.pending[z]);
            S.pendingCount[z] = 1;
        }
        a = EmptyAggBlk();
    }
    AggAdd(a, w);
    S.agg[z] = a;
}

// The window of a ZMW marked HQ at the end of `block`: blocks [b0, block].
__device__ __forceinline__ uint32_t WindowStart(const MetricSide& S, uint32_t block)
{
    return block + 1 >= S.lookback ? block + 1 - S.lookback : 0;
}

__device__ __forceinline__ const MetricBlk& RingAt(const MetricSide& S, uint32_t b, uint32_t z)
{
    return S.ring[(size_t)(b % S.lookback) * S.numZmw + z];
}

// Label runs of ZMW z's window, the first counted against "no label".
__device__ __forceinline__ uint32_t WindowRuns(const MetricSide& S, uint32_t block, uint32_t z)
{
    uint32_t n = 0;
    uint32_t cur = kNoActivity;
    for (uint32_t b = WindowStart(S, block); b <= block; ++b)
    {
        const uint32_t l = RingAt(S, b, z).label;
        if (l != cur)
        {
            ++n;
            cur = l;
        }
    }
    return n;
}

// mode 0: a block's end (newly = marked HQ now, hq = HQ before); 1: flush.
__global__ void MetricCountKernel(MetricSide S, const uint8_t* hq, const uint8_t* newly, uint32_t block, int mode,
                                  uint64_t* counts)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z == 0) counts[S.numZmw] = 0;
    if (z >= S.numZmw) return;
    uint32_t c = S.pendingCount[z];
    if (S.production)
    {
        if (mode == 1) c = S.agg[z].numFrames != 0 ? 1u : c;
        else if (newly[z] && !hq[z]) c = WindowRuns(S, block, z);
    }
    counts[z] = c;
}

__global__ void MetricWriteKernel(MetricSide S, const uint8_t* hq, const uint8_t* newly, uint32_t block, int mode,
                                  const uint64_t* offsets, hw_spider_metric_block* out)
{
    const uint32_t z = blockIdx.x * blockDim.x + threadIdx.x;
    if (z >= S.numZmw) return;
    hw_spider_metric_block* o = out + offsets[z];
    const uint64_t n = offsets[z + 1] - offsets[z];
    const bool pend = S.pendingCount[z] != 0;
    S.pendingCount[z] = 0;
    if (!S.production)
    {
        if (pend) *o = S.pending[z];
        return;
    }
    if (mode == 1)
    {
        const AggBlk a = S.agg[z];
        if (a.numFrames != 0) AggToSpider(a, *o);
        else if (pend) *o = S.pending[z];
        return;
    }
    if (pend)
    {
        *o = S.pending[z];
        return;
    }
    if (hq[z]) return;
    if (newly[z])
    {
        // the pre-HQ aggregate, then the window's label runs but the last
        // (only the first n of them: see WindowRuns)
        if (n > 0) AggToSpider(S.agg[z], o[0]);
        uint32_t b = WindowStart(S, block);
        AggBlk run = EmptyAggBlk();
        AggAdd(run, Widen(RingAt(S, b, z)));
        uint32_t cur = run.label;
        uint64_t k = 1;
        for (++b; b <= block; ++b)
        {
            const AggBlk e = Widen(RingAt(S, b, z));
            if (e.label != cur)
            {
                if (k < n) AggToSpider(run, o[k]);
                ++k;
                cur = e.label;
                run = EmptyAggBlk();
            }
            AggAdd(run, e);
        }
        AggBlk a = EmptyAggBlk();
        AggAdd(a, run);
        S.agg[z] = a;
        return;
    }
    // still pre-HQ: once the window is full its oldest block joins the
    // pre-HQ aggregate, and its slot starts the next block empty
    MetricBlk& slot = S.ring[(size_t)((block + 1) % S.lookback) * S.numZmw + z];
    if (block + 1 >= S.lookback)
    {
        AggBlk a = S.agg[z];
        AggAdd(a, Widen(slot));
        S.agg[z] = a;
    }
    slot = EmptyMetricBlk();
}

}   // namespace hwk
