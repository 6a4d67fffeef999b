// Multi-scale morphological baseliner for sm_100a.
//
// Restates TA/HostMultiScaleBaseliner.cpp:95-212, TA/TraceFilters.cpp:11-57,
// TA/BlockFilterStage.cpp:9-25 and DT/BaselinerStatAccumulator.cpp:39-53
// (TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes).
//
// Design: one thread per ZMW streams its chunk frame by frame.  The reference
// runs every filter stage in place over the whole block; because each stage is
// causal (output m depends on inputs m-w..m-1) and chunk lengths are multiples
// of the aggregate stride, the same values come out of a per-frame pipeline in
// which scale i is fed at frames t with t % cumStride_i == 0.  The final stage
// produces block i's lower/upper envelope at frame i*aggStride, exactly when the
// subtraction of that block starts, so the trace is read from HBM once and the
// baselined trace written once, with coalesced 64-byte warp accesses.
// Each stage window keeps the reference's van Herk/Gil-Werman state (ring of w
// values, holdover, counter) so the filter outputs are bit-identical.
#include "hw_device.cuh"

namespace hwk {

template <int FT> struct FSpec;
template <> struct FSpec<HW_FILTER_MULTISCALE_LARGE>  { static constexpr int n = 3; static constexpr int s[3] = {1, 2, 8}; static constexpr int w[3] = {11, 17, 61}; };
template <> struct FSpec<HW_FILTER_MULTISCALE_MEDIUM> { static constexpr int n = 3; static constexpr int s[3] = {1, 2, 8}; static constexpr int w[3] = {9, 17, 31}; };
template <> struct FSpec<HW_FILTER_MULTISCALE_SMALL>  { static constexpr int n = 3; static constexpr int s[3] = {1, 2, 8}; static constexpr int w[3] = {7, 17, 17}; };
template <> struct FSpec<HW_FILTER_TWOSCALE_LARGE>    { static constexpr int n = 2; static constexpr int s[3] = {2, 8, 1}; static constexpr int w[3] = {11, 61, 0}; };
template <> struct FSpec<HW_FILTER_TWOSCALE_MEDIUM>   { static constexpr int n = 2; static constexpr int s[3] = {2, 8, 1}; static constexpr int w[3] = {9, 31, 0}; };
template <> struct FSpec<HW_FILTER_TWOSCALE_SMALL>    { static constexpr int n = 2; static constexpr int s[3] = {2, 8, 1}; static constexpr int w[3] = {7, 17, 0}; };

template <int FT> struct FLayout
{
    using S = FSpec<FT>;
    static constexpr int nStages = 2 * S::n;           // per filter
    static constexpr int Width(int k) { return S::w[k / 2]; }
    // lower: erode, dilate, then erode/dilate; upper: dilate, erode, then erode/dilate
    static constexpr bool IsMax(bool upper, int k) { return (k < 2 && upper) ? (k == 0) : (k % 2 == 1); }
    static constexpr int RingTotal()
    {
        int t = 0;
        for (int k = 0; k < nStages; ++k) t += Width(k);
        return 2 * t;
    }
    static constexpr int RingOffset(bool upper, int k)
    {
        int t = upper ? RingTotal() / 2 : 0;
        for (int j = 0; j < k; ++j) t += Width(j);
        return t;
    }
    static constexpr int CumStride(int i)
    {
        int c = 1;
        for (int j = 0; j <= i; ++j) c *= S::s[j];
        return c;
    }
    static constexpr int AggStride() { return CumStride(S::n - 1); }
    // int16 state slots: rings, then (hold, counter) per stage, then latData, latRaw, masks
    static constexpr int SlotHold(bool upper, int k) { return RingTotal() + 2 * ((upper ? nStages : 0) + k); }
    static constexpr int SlotLatData() { return RingTotal() + 4 * nStages; }
    static constexpr int NumI16Slots() { return SlotLatData() + 3; }
};

// One van Herk/Gil-Werman window stage (TraceFilters.cpp:11-57 with the
// WindowBuffer of WindowBuffer.h: ring head == counter at all times).
template <int W, bool IsMax>
__device__ __forceinline__ int16_t StageStep(int16_t* ring, int16_t& hold, int16_t& counter, int16_t x)
{
    auto op = [](int16_t a, int16_t b) -> int16_t {
        return IsMax ? (a > b ? a : b) : (a < b ? a : b);
    };
    const int c = counter;
    int16_t s;
    if (c == 0)
    {
#pragma unroll 4
        for (int j = W - 1; j > 0; --j) ring[j - 1] = op(ring[j], ring[j - 1]);
        s = ring[W - 1];
    }
    else
    {
        s = op(hold, ring[c - 1]);
    }
    const int16_t front = ring[c];
    ring[c] = x;
    hold = s;
    counter = (int16_t)((c + 1 == W) ? 0 : c + 1);
    return op(s, front);
}

template <int FT, bool Upper, int Scale>
__device__ __forceinline__ int16_t RunScale(int16_t* ring, int16_t* hc, int16_t x)
{
    using Lay = FLayout<FT>;
    constexpr int k0 = 2 * Scale, k1 = 2 * Scale + 1;
    constexpr int o0 = Lay::RingOffset(Upper, k0) - (Upper ? Lay::RingTotal() / 2 : 0);
    constexpr int o1 = Lay::RingOffset(Upper, k1) - (Upper ? Lay::RingTotal() / 2 : 0);
    const int16_t y = StageStep<Lay::Width(k0), Lay::IsMax(Upper, k0)>(ring + o0, hc[2 * k0], hc[2 * k0 + 1], x);
    return StageStep<Lay::Width(k1), Lay::IsMax(Upper, k1)>(ring + o1, hc[2 * k1], hc[2 * k1 + 1], y);
}

// Feeds frame t (relative to the chunk) through one multi-scale filter; returns
// true and the envelope value when the last stage produced an output.
template <int FT, bool Upper>
__device__ __forceinline__ bool FeedFilter(int t, int16_t x, int16_t* ring, int16_t* hc, int16_t& out)
{
    using S = FSpec<FT>;
    using Lay = FLayout<FT>;
    if (t % Lay::CumStride(0) != 0) return false;
    int16_t y = RunScale<FT, Upper, 0>(ring, hc, x);
    if constexpr (S::n > 1)
    {
        if (t % Lay::CumStride(1) != 0) return false;
        y = RunScale<FT, Upper, 1>(ring, hc, y);
    }
    if constexpr (S::n > 2)
    {
        if (t % Lay::CumStride(2) != 0) return false;
        y = RunScale<FT, Upper, 2>(ring, hc, y);
    }
    out = y;
    return true;
}


template <int FT>
__global__ void __launch_bounds__(128) BaselinerKernel(BaselinerArgs a, KParams k)
{
    using Lay = FLayout<FT>;
    constexpr int RT = Lay::RingTotal();
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int nZmw = a.lanes * kLane;
    if (g >= nZmw) return;
    const int lane = g / kLane, z = g % kLane;

    // Load window state (rings are indexed dynamically: local memory).
    int16_t ringL[RT / 2], ringU[RT / 2];
    int16_t hcL[2 * Lay::nStages], hcU[2 * Lay::nStages];
#pragma unroll 8
    for (int i = 0; i < RT / 2; ++i)
    {
        ringL[i] = a.st16[(size_t)i * nZmw + g];
        ringU[i] = a.st16[(size_t)(i + RT / 2) * nZmw + g];
    }
#pragma unroll
    for (int s = 0; s < Lay::nStages; ++s)
    {
        hcL[2 * s] = a.st16[(size_t)Lay::SlotHold(false, s) * nZmw + g];
        hcL[2 * s + 1] = a.st16[(size_t)(Lay::SlotHold(false, s) + 1) * nZmw + g];
        hcU[2 * s] = a.st16[(size_t)Lay::SlotHold(true, s) * nZmw + g];
        hcU[2 * s + 1] = a.st16[(size_t)(Lay::SlotHold(true, s) + 1) * nZmw + g];
    }
    int16_t latData = a.st16[(size_t)Lay::SlotLatData() * nZmw + g];
    int16_t latRaw = a.st16[(size_t)(Lay::SlotLatData() + 1) * nZmw + g];
    const int16_t mbits = a.st16[(size_t)(Lay::SlotLatData() + 2) * nZmw + g];
    bool latL = mbits & 1, latH1 = (mbits >> 1) & 1, latH2 = (mbits >> 2) & 1;
    float uemaSum = a.st32[(size_t)0 * nZmw + g];
    float uemaWeight = a.st32[(size_t)1 * nZmw + g];
    float sigmaEma = a.st32[(size_t)2 * nZmw + g];

    // Per-chunk BaselinerStatAccumulator (fresh each chunk, offset 0).
    float c_m0 = 0, c_m1 = 0, c_m2 = 0, c_acm2 = 0;
    float fb0 = 0, fb1 = 0, fb2 = 0, fb3 = 0;
    float q0 = 0, q1 = 0, q2 = 0, q3 = 0;     // back buffer as a FIFO, q0 oldest
    int nAdded = 0;
    int16_t tmin = 32767, tmax = -32768;
    float b_m0 = 0, b_m1 = 0, b_m2 = 0, rawSum = 0;
    float g_m0 = 0, g_m1 = 0, g_m2 = 0;

    const int16_t* tr = a.trace + (size_t)lane * a.F * kLane + z;
    int16_t* out = a.out + (size_t)lane * a.F * kLane + z;
    const int16_t ped = (int16_t)k.pedestal;
    float sub = 0.0f;

    for (int t = 0; t < a.F; ++t)
    {
        const int16_t x = __ldg(tr + (size_t)t * kLane);
        int16_t lo = 0, up = 0;
        const bool haveL = FeedFilter<FT, false>(t, x, ringL, hcL, lo);
        FeedFilter<FT, true>(t, x, ringU, hcU, up);
        if (haveL)
        {
            // GetSmoothedBlEstimate (HostMultiScaleBaseliner.cpp:179-212)
            const int16_t lv = i16_wrap(lo - ped), uv = i16_wrap(up - ped);
            constexpr float minSigma = .288675135f;
            const float ma = k.meanEmaAlpha, sa = k.sigmaEmaAlpha;
            const float sigma = fmax_sse((float)i16_wrap(uv - lv) / k.cSigmaBias, minSigma);
            const float newSigmaEma = add_rn(mul_rn(sa, sigmaEma), mul_rn(1.0f - sa, sigma));
            const float blEst = add_rn(mul_rn(0.5f, (float)i16_wrap(uv + lv)), mul_rn(k.cMeanBias, newSigmaEma));
            const bool mask = (uemaWeight == 0.0f)
                            | (blEst - uemaSum / uemaWeight < k.jumpTolCoeff * sigmaEma);
            const float newWeight = add_rn(mul_rn(ma, uemaWeight), 1.0f - ma);
            const float newSum = add_rn(mul_rn(ma, uemaSum), mul_rn(1.0f - ma, blEst));
            uemaWeight = mask ? newWeight : uemaWeight;
            uemaSum = mask ? newSum : uemaSum;
            sigmaEma = mask ? newSigmaEma : sigmaEma;
            const float est = uemaSum / uemaWeight;
            sub = mul_rn(est, k.scaler);
            // AddSampleBackground (BaselinerStatAccumulator.cpp:56-60)
            const float bg = (float)to_i16_wrap(sub);
            g_m0 += 1.0f; g_m1 += bg; g_m2 = add_rn(g_m2, mul_rn(bg, bg));
        }
        const float rs = mul_rn((float)i16_wrap(x - ped), k.scaler);
        const int16_t bls = to_i16_wrap(rs - sub);
        out[(size_t)t * kLane] = bls;
        const int16_t raw = to_i16_wrap(rs);

        // AddToBaselineStats (HostMultiScaleBaseliner.cpp:148-176)
        const float thr = mul_rn(4.5f, sigmaEma);
        const bool hp1 = (float)bls < mul_rn(thr, k.scaler);
        const bool m = latH1 & latL & hp1;
        latL = (float)bls < mul_rn(thr, k.scaler);
        latH2 = latH1;
        latH1 = hp1;
        {
            // BaselinerStatAccumulator::AddSample(latRaw, latData, m)
            const float v = (float)latData;
            if (nAdded < 4)
            {
                if (nAdded == 0) fb0 = v; else if (nAdded == 1) fb1 = v; else if (nAdded == 2) fb2 = v; else fb3 = v;
            }
            c_acm2 = add_rn(c_acm2, mul_rn(q0, v));
            q0 = q1; q1 = q2; q2 = q3; q3 = v;
            ++nAdded;
            c_m0 += 1.0f; c_m1 += v; c_m2 = add_rn(c_m2, mul_rn(v, v));
            tmin = latData < tmin ? latData : tmin;
            tmax = latData > tmax ? latData : tmax;
            const float a0 = b_m0 + 1.0f, a1 = b_m1 + v, a2 = add_rn(b_m2, mul_rn(v, v));
            b_m0 = m ? a0 : b_m0; b_m1 = m ? a1 : b_m1; b_m2 = m ? a2 : b_m2;
            rawSum += (float)(m ? latRaw : (int16_t)0);
        }
        latRaw = raw;
        latData = bls;
    }

    // Store state.
#pragma unroll 8
    for (int i = 0; i < RT / 2; ++i)
    {
        a.st16[(size_t)i * nZmw + g] = ringL[i];
        a.st16[(size_t)(i + RT / 2) * nZmw + g] = ringU[i];
    }
#pragma unroll
    for (int s = 0; s < Lay::nStages; ++s)
    {
        a.st16[(size_t)Lay::SlotHold(false, s) * nZmw + g] = hcL[2 * s];
        a.st16[(size_t)(Lay::SlotHold(false, s) + 1) * nZmw + g] = hcL[2 * s + 1];
        a.st16[(size_t)Lay::SlotHold(true, s) * nZmw + g] = hcU[2 * s];
        a.st16[(size_t)(Lay::SlotHold(true, s) + 1) * nZmw + g] = hcU[2 * s + 1];
    }
    a.st16[(size_t)Lay::SlotLatData() * nZmw + g] = latData;
    a.st16[(size_t)(Lay::SlotLatData() + 1) * nZmw + g] = latRaw;
    a.st16[(size_t)(Lay::SlotLatData() + 2) * nZmw + g] = (int16_t)((latL ? 1 : 0) | (latH1 ? 2 : 0) | (latH2 ? 4 : 0));
    a.st32[(size_t)0 * nZmw + g] = uemaSum;
    a.st32[(size_t)1 * nZmw + g] = uemaWeight;
    a.st32[(size_t)2 * nZmw + g] = sigmaEma;

    // Per-chunk stats (GetState of the accumulator).
    hw_baseliner_stats& S = a.stats[lane];
    S.full_autocorr.basic_stats.offset[z] = 0.0f;
    S.full_autocorr.basic_stats.moment0[z] = c_m0;
    S.full_autocorr.basic_stats.moment1[z] = c_m1;
    S.full_autocorr.basic_stats.moment2[z] = c_m2;
    S.full_autocorr.moment2[z] = c_acm2;
    const int fbi = nAdded < 4 ? nAdded : 4;
    const int bbi = nAdded % 4;
    S.full_autocorr.fbuf[0][z] = fb0; S.full_autocorr.fbuf[1][z] = fb1;
    S.full_autocorr.fbuf[2][z] = fb2; S.full_autocorr.fbuf[3][z] = fb3;
    // bBuf[(bbi + j) % 4] holds the j-th oldest of the last four samples.
    const float qq[4] = {q0, q1, q2, q3};
#pragma unroll
    for (int j = 0; j < 4; ++j) S.full_autocorr.bbuf[(bbi + j) % 4][z] = qq[j];
    S.full_autocorr.bidx[0][z] = (uint8_t)fbi;
    S.full_autocorr.bidx[1][z] = (uint8_t)bbi;
    S.trace_min[z] = tmin;
    S.trace_max[z] = tmax;
    S.baseline_stats.offset[z] = 0.0f;
    S.baseline_stats.moment0[z] = b_m0;
    S.baseline_stats.moment1[z] = b_m1;
    S.baseline_stats.moment2[z] = b_m2;
    S.raw_baseline_sum[z] = rawSum;
    S.background_stats.offset[z] = 0.0f;
    S.background_stats.moment0[z] = g_m0;
    S.background_stats.moment1[z] = g_m1;
    S.background_stats.moment2[z] = g_m2;
}

template <int FT>
int BaselinerSlots16() { return FLayout<FT>::NumI16Slots(); }

int BaselinerNumSlots16(int ft)
{
    switch (ft)
    {
    case 0: return BaselinerSlots16<0>();
    case 1: return BaselinerSlots16<1>();
    case 2: return BaselinerSlots16<2>();
    case 3: return BaselinerSlots16<3>();
    case 4: return BaselinerSlots16<4>();
    case 5: return BaselinerSlots16<5>();
    }
    return -1;
}

cudaError_t LaunchBaseliner(int ft, const BaselinerArgs& a, const KParams& k, cudaStream_t s)
{
    const int threads = 128;
    const int blocks = (a.lanes * kLane + threads - 1) / threads;
    switch (ft)
    {
    case 0: BaselinerKernel<0><<<blocks, threads, 0, s>>>(a, k); break;
    case 1: BaselinerKernel<1><<<blocks, threads, 0, s>>>(a, k); break;
    case 2: BaselinerKernel<2><<<blocks, threads, 0, s>>>(a, k); break;
    case 3: BaselinerKernel<3><<<blocks, threads, 0, s>>>(a, k); break;
    case 4: BaselinerKernel<4><<<blocks, threads, 0, s>>>(a, k); break;
    case 5: BaselinerKernel<5><<<blocks, threads, 0, s>>>(a, k); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}   // namespace hwk
