// Baseline-statistics aggregation, trace histogram and model initialisation.
//
// Restates (TA = src/basecaller/basecaller/traceAnalysis, DT = .../dataTypes,
// CM = .../common):
//   TA/BaselineStatsAggregatorHost.cpp:37-45 + CM/AutocorrAccumulator.cpp:71-103
//   TA/TraceHistogramAccumHost.cpp:82-169, TA/EdgeFrameClassifier.h:72-94,
//   DT/UHistogramSimd.{h:199-229, cpp:51-97}
//   TA/DmeEmHost.cpp:872-925 (InitLaneDetModel)
// One thread per ZMW; lane structs are structure-of-arrays so every access is
// a coalesced row of 64 values.
#include "hw_device.cuh"

namespace hwk {

// ---- BaselinerStatAccumulator::Merge -------------------------------------

__global__ void AggResetKernel(hw_baseliner_stats* s, int lanes, LaneMap map)
{
    int l, z;
    if (!ZmwOf(map, lanes, l, z)) return;
    hw_baseliner_stats& S = s[l];
    hw_stat_accum_state* st[3] = {&S.full_autocorr.basic_stats, &S.baseline_stats, &S.background_stats};
    for (auto* p : st) { p->offset[z] = 0; p->moment0[z] = 0; p->moment1[z] = 0; p->moment2[z] = 0; }
    S.full_autocorr.moment2[z] = 0;
    for (int k = 0; k < 4; ++k) { S.full_autocorr.fbuf[k][z] = 0; S.full_autocorr.bbuf[k][z] = 0; }
    S.full_autocorr.bidx[0][z] = 0;
    S.full_autocorr.bidx[1][z] = 0;
    S.trace_min[z] = 32767;
    S.trace_max[z] = -32768;
    S.raw_baseline_sum[z] = 0;
}

__global__ void AggMergeKernel(hw_baseliner_stats* acc, const hw_baseliner_stats* in, int lanes, LaneMap map)
{
    int l, z;
    if (!ZmwOf(map, lanes, l, z)) return;
    hw_baseliner_stats& A = acc[l];
    const hw_baseliner_stats& B = in[l];
    auto mergeStat = [z](hw_stat_accum_state& a, const hw_stat_accum_state& b) {
        a.moment0[z] += b.moment0[z];
        a.moment1[z] += b.moment1[z];
        a.moment2[z] += b.moment2[z];
    };
    // AutocorrAccumulator::Merge
    mergeStat(A.full_autocorr.basic_stats, B.full_autocorr.basic_stats);
    float m2 = A.full_autocorr.moment2[z] + B.full_autocorr.moment2[z];
    const int tfbi = B.full_autocorr.bidx[0][z], tbbi = B.full_autocorr.bidx[1][z];
    const int fbi = A.full_autocorr.bidx[0][z], bbi = A.full_autocorr.bidx[1][z];
    const int n1 = 4 - tfbi;
    for (int k = 0; k < 4 - n1; ++k)
    {
        const int i = (bbi + k) % 4, j = (tbbi + n1 + k) % 4;
        m2 = add_rn(m2, mul_rn(A.full_autocorr.bbuf[i][z], B.full_autocorr.fbuf[k][z]));
        A.full_autocorr.bbuf[i][z] = B.full_autocorr.bbuf[j][z];
    }
    const int n2 = 4 - fbi;
    for (int k = 0; k < n2; ++k) A.full_autocorr.fbuf[fbi + k][z] = B.full_autocorr.fbuf[k][z];
    A.full_autocorr.moment2[z] = m2;
    A.full_autocorr.bidx[0][z] = (uint8_t)(fbi + n2);
    A.full_autocorr.bidx[1][z] = (uint8_t)((bbi + (4 - n1)) % 4);
    A.trace_min[z] = min(A.trace_min[z], B.trace_min[z]);
    A.trace_max[z] = max(A.trace_max[z], B.trace_max[z]);
    mergeStat(A.baseline_stats, B.baseline_stats);
    A.raw_baseline_sum[z] += B.raw_baseline_sum[z];
    mergeStat(A.background_stats, B.background_stats);
}

// StatAccumulator::Mean / Variance (CM/StatAccumulator.h:85-97)
__device__ __forceinline__ float StatMean(const hw_stat_accum_state& s, int z)
{
    return s.moment1[z] / s.moment0[z] + s.offset[z];
}

__device__ __forceinline__ float StatVariance(const hw_stat_accum_state& s, int z)
{
    const float m0 = s.moment0[z], m1 = s.moment1[z], m2 = s.moment2[z];
    float var = mul_rn(m1, m1) / m0;
    var = (m2 - var) / (m0 - 1.0f);
    var = fmax_sse(var, 0.0f);
    return (m0 > 1.0f) ? var : __int_as_float(0x7fffffff);
}

// ---- Histogram ------------------------------------------------------------

// UHistogramSimd ctor checks (UHistogramSimd.cpp:66-96).
__device__ __forceinline__ bool HistBoundsOk(float lo, float up, float bs)
{
    bool ok = !(lo >= up) && !(bs <= 0.0f);
    float prev = lo;
    for (int i = 1; i <= kBins; ++i)
    {
        const float si = add_rn(mul_rn(bs, (float)i), lo);
        ok &= !(prev == si);
        prev = si;
    }
    return ok;
}

__device__ __forceinline__ void HistClear(hw_lane_histogram& H, int z)
{
    H.outlier_count_low[z] = 0;
    H.outlier_count_high[z] = 0;
    for (int b = 0; b < kBins; ++b) H.bin_count[b][z] = 0;
}

// TraceHistogramAccumHost::ResetImpl(const BaselinerMetrics&), :96-126
__global__ void HistResetStatsKernel(hw_lane_histogram* hist, const hw_baseliner_stats* stats, int lanes,
                                     KParams k, int* err, LaneMap map)
{
    int l, z;
    if (!ZmwOf(map, lanes, l, z)) return;
    const hw_stat_accum_state& s = stats[l].baseline_stats;
    const bool suff = s.moment0[z] >= k.minFrameCount;
    const float mean = suff ? StatMean(s, z) : 0.0f;
    const float sigma = suff ? sqrtf(StatVariance(s, z)) : k.fallbackSigma;
    const float binSize = fmax_sse(mul_rn(k.binSizeCoeff, sigma), k.binSizeMin);
    const float lo = mean - mul_rn(4.0f, sigma);
    const float up = add_rn(lo, mul_rn(float(kBins), binSize));
    const float bs = (up - lo) / static_cast<float>(kBins);
    hw_lane_histogram& H = hist[l];
    H.low_bound[z] = lo;
    H.bin_size[z] = bs;
    HistClear(H, z);
    if (!HistBoundsOk(lo, up, bs)) atomicCAS(err, 0, HW_ERR_NUMERIC);
}

// TraceHistogramAccumHost::ResetImpl(const UnifiedCudaArray<LaneHistBounds>&), :82-94
__global__ void HistResetBoundsKernel(hw_lane_histogram* hist, const hw_lane_hist_bounds* b, int lanes, int* err, LaneMap map)
{
    int l, z;
    if (!ZmwOf(map, lanes, l, z)) return;
    const float lo = b[l].lower_bounds[z], up = b[l].upper_bounds[z];
    const float bs = (up - lo) / static_cast<float>(kBins);
    hist[l].low_bound[z] = lo;
    hist[l].bin_size[z] = bs;
    HistClear(hist[l], z);
    if (!HistBoundsOk(lo, up, bs)) atomicCAS(err, 0, HW_ERR_NUMERIC);
}

// Edge classifier state per ZMW: prev frame and a two-deep baseline history.
struct EdgeState
{
    int16_t* prev;      // [nZmw]
    uint8_t* bits;      // [nZmw]: bit0 isBl(t-1), bit1 isBl(t-2), bits 2-3 count (0..2)
};

constexpr int kHistLanesPerBlock = 1;

constexpr int kHistBatch = 8;
constexpr int kHistPairBatch = 4;   // frames of each half loaded ahead

// Bin of v = (x - lower) / binSize as floor_cast_i32(v) classifies it:
// -1 for every value that floor_cast_i32 makes negative (v < 0, NaN, and
// v >= 2^31, which it turns into INT_MIN), kBins for 300 <= v < 2^31, else
// floor(v).  For 0 <= v < 300, v + 2^23 rounded down is exactly 2^23 +
// floor(v) (the spacing of floats in [2^23, 2^24) is 1), so the floor
// costs one add on the FMA pipe instead of a round and a conversion.
__device__ __forceinline__ int HistBin(float v)
{
    if (v >= 0.0f && v < (float)kBins) return __float_as_int(__fadd_rd(v, 8388608.0f)) - 0x4B000000;
    return (v >= (float)kBins && v < 2147483648.0f) ? kBins : -1;
}

// int16 -> float, exactly: 1.5 x 2^23 + x has the bit pattern 0x4B400000 + x.
__device__ __forceinline__ float I16ToFloat(int16_t x) { return __int_as_float(0x4B400000 + (int)x) - 12582912.0f; }

// AddBlock (TraceHistogramAccumHost.cpp:140-169): edge scrubbing with the fp16
// baseline mode, then UHistogramSimd::AddDatum.  Counts of the lane are held
// in shared memory for the chunk (one u16 per bin and ZMW; each thread only
// touches its own ZMW's column, so no atomics are needed).
__global__ void __launch_bounds__(kLane * kHistLanesPerBlock)
HistAddKernel(hw_lane_histogram* hist, EdgeState es, const int16_t* traces, int frames,
              const hw_lane_model* models, int lanes, LaneMap map)
{
    extern __shared__ uint16_t histSmem[];
    auto cnt = reinterpret_cast<uint16_t (*)[kBins + 1][kLane]>(histSmem);
    const int ll = threadIdx.x / kLane, z = threadIdx.x % kLane;
    const int li = blockIdx.x * kHistLanesPerBlock + ll;
    static_assert(kHistLanesPerBlock == 1, "the block-wide copies below need one lane per block");
    if (li >= map.Lanes(lanes)) return;    // the whole block (one lane) returns together
    const int l = map.Lane(li);
    if (map.On()) frames = map.Pool(l).F;
    const int g = l * kLane + z;
    hw_lane_histogram& H = hist[l];
    // The lane's counts [300][64] u16 are one contiguous 38,400-byte block in
    // global and in shared memory: every thread issues its share of 16-byte
    // asynchronous copies, all in flight together, then the block waits once.
    constexpr int kChunks = kBins * kLane * 2 / 16;
    {
        const char* src = reinterpret_cast<const char*>(&H.bin_count[0][0]);
        const uint32_t dst = (uint32_t)__cvta_generic_to_shared(&cnt[ll][0][0]);
        for (int c = threadIdx.x; c < kChunks; c += blockDim.x)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst + 16 * c), "l"(src + 16 * c));
        asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
        __syncthreads();
    }
    uint16_t nLow = H.outlier_count_low[z], nHigh = H.outlier_count_high[z];
    const float lower = H.low_bound[z], binSize = H.bin_size[z];
    const float bm = h2f(models[l].baseline.means[z]);
    const float bv = h2f(models[l].baseline.vars[z]);
    const int16_t thr = i16_wrap(cvt_rn_i32(add_rn(mul_rn(2.0f, sqrtf(bv)), bm)));
    int16_t prev = es.prev[g];
    uint8_t bits = es.bits[g];
    bool b1 = bits & 1, b2 = (bits >> 1) & 1;
    int n = (bits >> 2) & 3;
    const int16_t* tr = traces + map.Block(l, frames) + z;
    auto step = [&](int16_t x) {
        const bool isBl = x < thr;
        const bool edge = (n == 2) ? (isBl ^ b2) : true;
        const float xv = I16ToFloat(prev);
        prev = x;
        b2 = b1; b1 = isBl; n = (n < 2) ? n + 1 : 2;
        const bool sel = !edge;
        int bin = HistBin((xv - lower) / binSize);
        const bool mLow = sel & (bin < 0);
        const bool mHigh = sel & (bin >= kBins);
        nLow = (uint16_t)(nLow + (mLow ? 1 : 0));
        nHigh = (uint16_t)(nHigh + (mHigh ? 1 : 0));
        if ((!sel) | mLow | mHigh) bin = kBins;
        cnt[ll][bin][z] = (uint16_t)(cnt[ll][bin][z] + 1);
    };
    int f = 0;
    if (frames >= 4 * kHistPairBatch && frames % (4 * kHistPairBatch) == 0)
    {
        // Two halves of the chunk at once, each with its own edge-classifier
        // state: the classifier looks back two frames only, so the second
        // half starts exactly from frames S-2 and S-1.  Two independent
        // divide / count chains are in flight; when both frames land in the
        // same bin the count is bumped by two once, so the counts equal the
        // one-stream ones.  Loads run a batch ahead in alternating registers.
        const int S = frames / 2;
        const int16_t xm2 = __ldg(tr + (size_t)(S - 2) * kLane), xm1 = __ldg(tr + (size_t)(S - 1) * kLane);
        int16_t prevB = xm1;
        bool b1B = xm1 < thr, b2B = xm2 < thr;
        uint16_t nLowB = 0, nHighB = 0;
        auto binOf = [&](int16_t x, int16_t& pv, bool& c1, bool& c2, int& cn, uint16_t& lo, uint16_t& hi) {
            const bool isBl = x < thr;
            const bool edge = (cn == 2) ? (isBl ^ c2) : true;
            const float xv = I16ToFloat(pv);
            pv = x;
            c2 = c1; c1 = isBl; cn = (cn < 2) ? cn + 1 : 2;
            const bool sel = !edge;
            int bin = HistBin((xv - lower) / binSize);
            const bool mLow = sel & (bin < 0);
            const bool mHigh = sel & (bin >= kBins);
            lo = (uint16_t)(lo + (mLow ? 1 : 0));
            hi = (uint16_t)(hi + (mHigh ? 1 : 0));
            if ((!sel) | mLow | mHigh) bin = kBins;
            return bin;
        };
        int nB = 2;
        auto pair = [&](int16_t xA, int16_t xB) {
            const int ba = binOf(xA, prev, b1, b2, n, nLow, nHigh);
            const int bb = binOf(xB, prevB, b1B, b2B, nB, nLowB, nHighB);
            const uint16_t ca = cnt[ll][ba][z], cb = cnt[ll][bb][z];
            if (ba == bb)
                cnt[ll][ba][z] = (uint16_t)(ca + 2);
            else
            {
                cnt[ll][ba][z] = (uint16_t)(ca + 1);
                cnt[ll][bb][z] = (uint16_t)(cb + 1);
            }
        };
        int16_t aA[kHistPairBatch], aB[kHistPairBatch], bA[kHistPairBatch], bB[kHistPairBatch];
#pragma unroll
        for (int j = 0; j < kHistPairBatch; ++j)
        {
            aA[j] = __ldg(tr + (size_t)j * kLane);
            aB[j] = __ldg(tr + (size_t)(S + j) * kLane);
        }
        int i = 0;
        for (; i + 2 * kHistPairBatch <= S; i += 2 * kHistPairBatch)
        {
#pragma unroll
            for (int j = 0; j < kHistPairBatch; ++j)
            {
                bA[j] = __ldg(tr + (size_t)(i + kHistPairBatch + j) * kLane);
                bB[j] = __ldg(tr + (size_t)(S + i + kHistPairBatch + j) * kLane);
            }
#pragma unroll
            for (int j = 0; j < kHistPairBatch; ++j) pair(aA[j], aB[j]);
            if (i + 3 * kHistPairBatch <= S)
            {
#pragma unroll
                for (int j = 0; j < kHistPairBatch; ++j)
                {
                    aA[j] = __ldg(tr + (size_t)(i + 2 * kHistPairBatch + j) * kLane);
                    aB[j] = __ldg(tr + (size_t)(S + i + 2 * kHistPairBatch + j) * kLane);
                }
            }
#pragma unroll
            for (int j = 0; j < kHistPairBatch; ++j) pair(bA[j], bB[j]);
        }
        // S is a multiple of 2 x kHistPairBatch: nothing is left over
        nLow = (uint16_t)(nLow + nLowB);
        nHigh = (uint16_t)(nHigh + nHighB);
        prev = prevB;
        b1 = b1B;
        b2 = b2B;
        n = nB;
        f = frames;
    }
    else
    {
        // Trace values in two register batches of 8 frames that alternate:
        // batch A is refilled while batch B is binned and vice versa, so
        // loads are a batch ahead and no register is copied while its load
        // is in flight.
        int16_t xa[kHistBatch], xb[kHistBatch];
        if (frames >= 2 * kHistBatch)
        {
#pragma unroll
            for (int j = 0; j < kHistBatch; ++j) xa[j] = __ldg(tr + (size_t)j * kLane);
        }
        for (; f + 2 * kHistBatch <= frames; f += 2 * kHistBatch)
        {
#pragma unroll
            for (int j = 0; j < kHistBatch; ++j) xb[j] = __ldg(tr + (size_t)(f + kHistBatch + j) * kLane);
#pragma unroll
            for (int j = 0; j < kHistBatch; ++j) step(xa[j]);
            if (f + 3 * kHistBatch <= frames)
            {
#pragma unroll
                for (int j = 0; j < kHistBatch; ++j) xa[j] = __ldg(tr + (size_t)(f + 2 * kHistBatch + j) * kLane);
            }
#pragma unroll
            for (int j = 0; j < kHistBatch; ++j) step(xb[j]);
        }
    }
    for (; f < frames; ++f) step(__ldg(tr + (size_t)f * kLane));
    __syncthreads();
    {
        uint4* dst = reinterpret_cast<uint4*>(&H.bin_count[0][0]);
        const uint4* src = reinterpret_cast<const uint4*>(&cnt[ll][0][0]);
        for (int c = threadIdx.x; c < kChunks; c += blockDim.x) dst[c] = src[c];
    }
    H.outlier_count_low[z] = nLow;
    H.outlier_count_high[z] = nHigh;
    es.prev[g] = prev;
    es.bits[g] = (uint8_t)((b1 ? 1 : 0) | (b2 ? 2 : 0) | (n << 2));
}

// ---- DmeEmHost::InitLaneDetModel (DmeEmHost.cpp:872-925) ------------------

__global__ void InitModelsKernel(hw_lane_model* models, const hw_baseliner_stats* stats, int lanes, KParams k,
                                 int fixedModel, float fixedMean, float fixedVar, LaneMap map)
{
    int l, z;
    if (!ZmwOf(map, lanes, l, z)) return;
    hw_lane_model& m = models[l];
    if (fixedModel)
    {
        // FixedModelBatchAnalyzer (BatchAnalyzer.cpp:77-101) sets means and
        // variances only; weights and confidence keep their values.
        return;
    }
    const hw_stat_accum_state& bl = stats[l].baseline_stats;
    const float blWeight = bl.moment0[z] / stats[l].full_autocorr.basic_stats.moment0[z];
    float blMean = StatMean(bl, z);
    float blVar = StatVariance(bl, z);
    blMean = isnan(blMean) ? 0.0f : blMean;
    blVar = isnan(blVar) ? 100.0f : blVar;
    blVar = fmin_sse(fmax_sse(blVar, k.blVarMin), k.blVarMax);
    m.confidence[z] = f2h(0.1f);
    m.baseline.weights[z] = f2h(blWeight);
    m.baseline.means[z] = f2h(blMean);
    m.baseline.vars[z] = f2h(blVar);
    const float amw = (1.0f - blWeight) / (float)kAnalogs;
    const float refSignal = mul_rn(k.refSnr, sqrtf(blVar));
    for (int a = 0; a < kAnalogs; ++a)
    {
        m.analogs[a].weights[z] = f2h(amw);
        const float aMean = fmax_sse(0.0f, add_rn(blMean, mul_rn(k.relAmp[a], refSignal)));
        m.analogs[a].means[z] = f2h(aMean);
        m.analogs[a].vars[z] = f2h(SignalCovar(k, k.cv2[a], aMean, blVar));
    }
}

// ---- launchers -------------------------------------------------------------

static inline int Blocks(int lanes, int threads) { return (lanes * kLane + threads - 1) / threads; }

cudaError_t LaunchAggReset(hw_baseliner_stats* s, int lanes, cudaStream_t st, const LaneMap& map)
{
    if (map.Lanes(lanes) == 0) return cudaSuccess;
    AggResetKernel<<<Blocks(map.Lanes(lanes), 256), 256, 0, st>>>(s, lanes, map);
    return cudaGetLastError();
}

cudaError_t LaunchAggMerge(hw_baseliner_stats* acc, const hw_baseliner_stats* in, int lanes, cudaStream_t st,
                           const LaneMap& map)
{
    if (map.Lanes(lanes) == 0) return cudaSuccess;
    AggMergeKernel<<<Blocks(map.Lanes(lanes), 256), 256, 0, st>>>(acc, in, lanes, map);
    return cudaGetLastError();
}

cudaError_t LaunchHistResetStats(hw_lane_histogram* h, const hw_baseliner_stats* s, int lanes, const KParams& k,
                                 int* err, cudaStream_t st, const LaneMap& map)
{
    if (map.Lanes(lanes) == 0) return cudaSuccess;
    HistResetStatsKernel<<<Blocks(map.Lanes(lanes), 128), 128, 0, st>>>(h, s, lanes, k, err, map);
    return cudaGetLastError();
}

cudaError_t LaunchHistResetBounds(hw_lane_histogram* h, const hw_lane_hist_bounds* b, int lanes, int* err,
                                  cudaStream_t st)
{
    HistResetBoundsKernel<<<Blocks(lanes, 128), 128, 0, st>>>(h, b, lanes, err, LaneMap{});
    return cudaGetLastError();
}

cudaError_t LaunchHistAdd(hw_lane_histogram* h, int16_t* prev, uint8_t* bits, const int16_t* traces, int frames,
                          const hw_lane_model* models, int lanes, cudaStream_t st, const LaneMap& map)
{
    EdgeState es{prev, bits};
    const int n = map.Lanes(lanes);
    if (n == 0) return cudaSuccess;
    const int blocks = (n + kHistLanesPerBlock - 1) / kHistLanesPerBlock;
    const size_t smem = sizeof(uint16_t) * kHistLanesPerBlock * (kBins + 1) * kLane;
    static bool attrSet = false;
    if (!attrSet)
    {
        cudaError_t e = cudaFuncSetAttribute(HistAddKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attrSet = true;
    }
    HistAddKernel<<<blocks, kLane * kHistLanesPerBlock, smem, st>>>(h, es, traces, frames, models, lanes, map);
    return cudaGetLastError();
}

cudaError_t LaunchInitModels(hw_lane_model* m, const hw_baseliner_stats* s, int lanes, const KParams& k,
                             cudaStream_t st, const LaneMap& map)
{
    if (map.Lanes(lanes) == 0) return cudaSuccess;
    InitModelsKernel<<<Blocks(map.Lanes(lanes), 128), 128, 0, st>>>(m, s, lanes, k, 0, 0.0f, 0.0f, map);
    return cudaGetLastError();
}

}   // namespace hwk
