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
#include <type_traits>

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
    static constexpr int kSmemMaxWidth = 17;           // wider windows stay in global memory
    static constexpr int Width(int k) { return S::w[k / 2]; }
    // lower: erode, dilate, then erode/dilate; upper: dilate, erode, then erode/dilate
    static constexpr bool IsMax(bool upper, int k) { return (k < 2 && upper) ? (k == 0) : (k % 2 == 1); }
    static constexpr bool InSmem(int k) { return Width(k) <= kSmemMaxWidth; }
    static constexpr int Idx(bool upper, int k) { return (upper ? nStages : 0) + k; }   // 0 .. 2*nStages-1
    // Every stage keeps S[W] (suffix extrema of the previous block) and B[W]
    // (inputs of the current block) in shared or global memory.
    static constexpr int SmemSlots()
    {
        int t = 0;
        for (int k = 0; k < nStages; ++k) if (InSmem(k)) t += 2 * Width(k);
        return 2 * t;
    }
    static constexpr int Offset(bool upper, int k)   // within its storage (smem or global)
    {
        int t = 0;
        for (int u = 0; u < 2; ++u)
            for (int j = 0; j < nStages; ++j)
            {
                if (u == (upper ? 1 : 0) && j == k) return t;
                if (InSmem(j) == InSmem(k)) t += 2 * Width(j);
            }
        return t;
    }
    static constexpr int NumGlobalStages()
    {
        int t = 0;
        for (int k = 0; k < nStages; ++k) if (!InSmem(k)) ++t;
        return 2 * t;
    }
    // index of a global stage among the global stages (lower first)
    static constexpr int GIdx(bool upper, int k)
    {
        int t = 0;
        for (int u = 0; u < 2; ++u)
            for (int j = 0; j < nStages; ++j)
            {
                if (u == (upper ? 1 : 0) && j == k) return t;
                if (!InSmem(j)) ++t;
            }
        return t;
    }
    static constexpr int GlobalRingSlots()
    {
        int t = 0;
        for (int k = 0; k < nStages; ++k) if (!InSmem(k)) t += 2 * Width(k);
        return 2 * t;
    }
    static constexpr int CumStride(int i)
    {
        int c = 1;
        for (int j = 0; j <= i; ++j) c *= S::s[j];
        return c;
    }
    static constexpr int AggStride() { return CumStride(S::n - 1); }
    // int16 state: smem-resident arrays, global-resident arrays, then (P, c)
    // per stage, then latData, latRaw, masks.
    static constexpr int SlotSmem() { return 0; }
    static constexpr int SlotGlobal() { return SmemSlots(); }
    static constexpr int SlotPC(bool upper, int k) { return SmemSlots() + GlobalRingSlots() + 2 * Idx(upper, k); }
    static constexpr int SlotLatData() { return SmemSlots() + GlobalRingSlots() + 4 * nStages; }
    static constexpr int NumI16Slots() { return SlotLatData() + 3; }
};

// One van Herk/Gil-Werman window stage.  The output for each input is the
// extremum of the W previous inputs (TraceFilters.cpp:11-57 with the window
// state of WindowBuffer.h; the initial window holds W zeros).  The state is
// the suffix extrema S of the previous block of W inputs, the running
// extremum P of the current block and the current block's inputs B; the
// output at block position c is op(S[c], P).  `base` points at S[0] of this
// thread and `stride` separates consecutive array elements.
template <int W, bool IsMax>
__device__ __forceinline__ int16_t StageStep(int16_t* base, int stride, int16_t& P, int16_t& counter, int16_t x)
{
    auto op = [](int16_t a, int16_t b) -> int16_t {
        return IsMax ? (a > b ? a : b) : (a < b ? a : b);
    };
    int16_t* S = base;
    int16_t* B = base + W * stride;
    const int c = counter;
    const int16_t y = op(S[c * stride], P);
    B[c * stride] = x;
    P = op(P, x);
    if (c + 1 == W)
    {
        // New suffix extrema of the completed block.
        int16_t acc = x;
        S[(W - 1) * stride] = acc;
#pragma unroll 1
        for (int j = W - 2; j >= 0; --j)
        {
            acc = op(B[j * stride], acc);
            S[j * stride] = acc;
        }
        P = IsMax ? (int16_t)-32768 : (int16_t)32767;
        counter = 0;
    }
    else
    {
        counter = (int16_t)(c + 1);
    }
    return y;
}

// Global-memory window stage with S[counter] held in a register, loaded one
// call ahead of its use (S changes only when a block completes), so the
// stage never waits for memory on its critical path.  At a block's end the
// inputs are read in batches of 4 before the batch's results are stored, so
// the loads overlap instead of each waiting behind the previous store.
template <int W, bool IsMax>
__device__ __forceinline__ int16_t StageStepG(int16_t* base, int stride, int16_t& P, int16_t& counter,
                                              int16_t& sNext, int16_t x)
{
    auto op = [](int16_t a, int16_t b) -> int16_t {
        return IsMax ? (a > b ? a : b) : (a < b ? a : b);
    };
    int16_t* S = base;
    int16_t* B = base + W * stride;
    const int c = counter;
    const int16_t y = op(sNext, P);
    B[c * stride] = x;
    P = op(P, x);
    if (c + 1 == W)
    {
        int16_t acc = x;
        S[(W - 1) * stride] = acc;
        constexpr int kBatch = 4;
#pragma unroll 1
        for (int j0 = W - 2; j0 >= 0; j0 -= kBatch)
        {
            int16_t b[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (j0 - q >= 0) b[q] = B[(j0 - q) * stride];
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (j0 - q >= 0)
                {
                    acc = op(b[q], acc);
                    S[(j0 - q) * stride] = acc;
                }
        }
        sNext = acc;      // S[0]
        P = IsMax ? (int16_t)-32768 : (int16_t)32767;
        counter = 0;
    }
    else
    {
        counter = (int16_t)(c + 1);
        sNext = S[(c + 1) * stride];
    }
    return y;
}

struct StageMem
{
    int16_t* smem;     // this thread's column in shared memory
    int sstride;       // blockDim.x
    int16_t* gmem;     // this ZMW's column of the global-resident arrays
    int gstride;       // nZmw
    int16_t* sNext;    // per global stage: S[counter], loaded ahead
};

template <int FT, bool Upper, int K>
__device__ __forceinline__ int16_t Stage(const StageMem& m, int16_t* pc, int16_t x)
{
    using Lay = FLayout<FT>;
    constexpr int W = Lay::Width(K);
    constexpr int off = Lay::Offset(Upper, K);
    constexpr int i = Lay::Idx(Upper, K);
    if constexpr (Lay::InSmem(K))
        return StageStep<W, Lay::IsMax(Upper, K)>(m.smem + off * m.sstride, m.sstride, pc[2 * i], pc[2 * i + 1], x);
    else
        return StageStepG<W, Lay::IsMax(Upper, K)>(m.gmem + (size_t)off * m.gstride, m.gstride, pc[2 * i],
                                                   pc[2 * i + 1], m.sNext[Lay::GIdx(Upper, K)], x);
}

// sNext of every global-memory stage of one filter from the saved state
// (compile-time recursion: the stage layout tables are host constants).
template <int FT, bool Upper, int K>
__device__ __forceinline__ void LoadSNext(const StageMem& m, const int16_t* pc, int nZmw)
{
    using Lay = FLayout<FT>;
    if constexpr (K < Lay::nStages)
    {
        if constexpr (!Lay::InSmem(K))
        {
            constexpr int i = Lay::Idx(Upper, K);
            constexpr int off = Lay::Offset(Upper, K);
            m.sNext[Lay::GIdx(Upper, K)] = m.gmem[((size_t)off + (size_t)pc[2 * i + 1]) * (size_t)nZmw];
        }
        LoadSNext<FT, Upper, K + 1>(m, pc, nZmw);
    }
}

template <int FT, bool Upper, int Scale>
__device__ __forceinline__ int16_t RunScale(const StageMem& m, int16_t* pc, int16_t x)
{
    const int16_t y = Stage<FT, Upper, 2 * Scale>(m, pc, x);
    return Stage<FT, Upper, 2 * Scale + 1>(m, pc, y);
}

// Feeds one frame through one multi-scale filter; returns true and the
// envelope value when the last stage produced an output.  Cumulative strides
// are 1, 2 or 16 and chunks are multiples of 16 frames, so the scales that
// run depend only on the frame's phase within its 16-frame block:
// Phase 0 = first frame of the block, 1 = other even frames, 2 = odd frames.
template <int Phase>
__host__ __device__ constexpr bool ScaleRuns(int cumStride)
{
    return cumStride == 1 || (cumStride == 2 && Phase <= 1) || (cumStride == 16 && Phase == 0);
}

template <int FT, bool Upper, int Phase>
__device__ __forceinline__ bool FeedFilter(int16_t x, const StageMem& m, int16_t* pc, int16_t& out)
{
    using S = FSpec<FT>;
    using Lay = FLayout<FT>;
    static_assert(Lay::CumStride(0) <= 2 && (S::n < 2 || Lay::CumStride(1) <= 16) && Lay::AggStride() == 16,
                  "phase scheme needs cumulative strides 1|2, 2, 16");
    if constexpr (!ScaleRuns<Phase>(Lay::CumStride(0))) return false;
    int16_t y = RunScale<FT, Upper, 0>(m, pc, x);
    if constexpr (S::n > 1)
    {
        if constexpr (!ScaleRuns<Phase>(Lay::CumStride(1))) return false;
        y = RunScale<FT, Upper, 1>(m, pc, y);
    }
    if constexpr (S::n > 2)
    {
        if constexpr (!ScaleRuns<Phase>(Lay::CumStride(2))) return false;
        y = RunScale<FT, Upper, 2>(m, pc, y);
    }
    out = y;
    return true;
}

// Initial filter state: every window holds W zeros (S = 0), the current block
// is empty (P = identity of the stage's operation, counter 0).
template <int FT>
__global__ void BaselinerInitKernel(int16_t* st16, float* st32, int lanes)
{
    using Lay = FLayout<FT>;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    const int nZmw = lanes * kLane;
    if (g >= nZmw) return;
    for (int i = 0; i < Lay::NumI16Slots(); ++i) st16[(size_t)i * nZmw + g] = 0;
    for (int u = 0; u < 2; ++u)
        for (int k = 0; k < Lay::nStages; ++k)
            st16[(size_t)Lay::SlotPC(u == 1, k) * nZmw + g] = Lay::IsMax(u == 1, k) ? (int16_t)-32768 : (int16_t)32767;
    st32[(size_t)0 * nZmw + g] = 0.0f;
    st32[(size_t)1 * nZmw + g] = 0.0f;
    st32[(size_t)2 * nZmw + g] = 2.0f;     // blSigmaEma_ initial value
}

template <int FT, typename TIn, bool Mapped>
__global__ void __launch_bounds__(64, 7) BaselinerKernel(BaselinerArgs a, KParams k)
{
    using Lay = FLayout<FT>;
    LaneMap map = a.map;
    if (!Mapped) map.list = nullptr;      // the single-pool variant compiles without the lane list
    const int gl = blockIdx.x * blockDim.x + threadIdx.x;
    const int nZmw = a.lanes * kLane;
    if (gl >= map.Lanes(a.lanes) * kLane) return;   // whole lanes only: the block is one lane
    const int z = gl % kLane;
    const int lane = map.Lane(gl / kLane);
    const int g = lane * kLane + z;
    const PoolStep* ps = map.On() ? &map.Pool(lane) : nullptr;
    const int F = ps ? ps->F : a.F;

    // Window state: narrow windows in shared memory (one column per thread),
    // wide ones used in place in global memory.
    extern __shared__ int16_t blSmem[];
    constexpr int SS = Lay::SmemSlots();
    constexpr int NG = Lay::NumGlobalStages() > 0 ? Lay::NumGlobalStages() : 1;
    int16_t sNext[NG];
    const StageMem mem{blSmem + threadIdx.x, (int)blockDim.x, a.st16 + (size_t)Lay::SlotGlobal() * nZmw + g, nZmw,
                       sNext};
#pragma unroll 32
    for (int i = 0; i < SS; ++i) blSmem[i * blockDim.x + threadIdx.x] = a.st16[(size_t)(Lay::SlotSmem() + i) * nZmw + g];
    int16_t pc[4 * Lay::nStages];
#pragma unroll
    for (int i = 0; i < 2 * Lay::nStages; ++i)
    {
        const bool up = i >= Lay::nStages;
        const int k = up ? i - Lay::nStages : i;
        pc[2 * i] = a.st16[(size_t)Lay::SlotPC(up, k) * nZmw + g];
        pc[2 * i + 1] = a.st16[(size_t)(Lay::SlotPC(up, k) + 1) * nZmw + g];
    }
    // S[counter] of every global stage
    LoadSNext<FT, false, 0>(mem, pc, nZmw);
    LoadSNext<FT, true, 0>(mem, pc, nZmw);
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

    const TIn* tr;
    const size_t inOff = ps ? (size_t)(lane - ps->lane0) * F * kLane : (size_t)lane * F * kLane;
    if constexpr (std::is_same_v<TIn, uint8_t>) tr = (ps ? ps->trace8 : a.trace8) + inOff + z;
    else tr = (ps ? ps->trace : a.trace) + inOff + z;
    int16_t* out = a.out + map.Block(lane, F) + z;
    const int16_t ped = (int16_t)k.pedestal;
    float sub = 0.0f;

    // Frames go in blocks of 16 (the aggregate stride): the first frame of a
    // block, the other even frames and the odd frames each get their own
    // specialisation of the frame body, with the trace loaded two frames ahead.
    // Even frames take their value from xEven and odd frames from xOdd, each
    // refilled right after use: no register is copied while its load is in
    // flight (a rotation xn0 = xn1 would wait for the newest load every frame).
    static_assert(Lay::AggStride() == 16, "block size must be the aggregate stride");
    int16_t xEven = (int16_t)__ldg(tr), xOdd = (int16_t)__ldg(tr + kLane);
    auto frame = [&](auto phaseTag, int t) {
        constexpr int Ph = decltype(phaseTag)::value;
        int16_t& slot = (Ph == 2) ? xOdd : xEven;      // phase 2 = odd frames
        const int16_t x = slot;
        if (t + 2 < F) slot = (int16_t)__ldg(tr + (size_t)(t + 2) * kLane);
        int16_t lo = 0, up = 0;
        const bool haveL = FeedFilter<FT, false, Ph>(x, mem, pc, lo);
        FeedFilter<FT, true, Ph>(x, mem, pc, up);
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
    };
#pragma unroll 1
    for (int t0 = 0; t0 < F; t0 += 16)
    {
        frame(std::integral_constant<int, 0>{}, t0);
#pragma unroll 1
        for (int j = 1; j < 16; j += 2)
        {
            frame(std::integral_constant<int, 2>{}, t0 + j);
            if (j + 1 < 16) frame(std::integral_constant<int, 1>{}, t0 + j + 1);
        }
    }

    // Store state.
#pragma unroll 8
    for (int i = 0; i < SS; ++i) a.st16[(size_t)(Lay::SlotSmem() + i) * nZmw + g] = blSmem[i * blockDim.x + threadIdx.x];
#pragma unroll
    for (int i = 0; i < 2 * Lay::nStages; ++i)
    {
        const bool up = i >= Lay::nStages;
        const int k = up ? i - Lay::nStages : i;
        a.st16[(size_t)Lay::SlotPC(up, k) * nZmw + g] = pc[2 * i];
        a.st16[(size_t)(Lay::SlotPC(up, k) + 1) * nZmw + g] = pc[2 * i + 1];
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

template <int FT, typename TIn, bool Mapped>
cudaError_t LaunchBaselinerT3(const BaselinerArgs& a, const KParams& k, cudaStream_t s)
{
    const int threads = kLane;
    const size_t smem = sizeof(int16_t) * FLayout<FT>::SmemSlots() * threads;
    // the shared-memory limit is a per-device attribute of the kernel: set it
    // once on each device
    static bool attrSet[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !attrSet[dev])
    {
        e = cudaFuncSetAttribute(BaselinerKernel<FT, TIn, Mapped>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attrSet[dev] = true;
    }
    const int blocks = a.map.Lanes(a.lanes);
    if (blocks == 0) return cudaSuccess;
    BaselinerKernel<FT, TIn, Mapped><<<blocks, threads, smem, s>>>(a, k);
    return cudaGetLastError();
}

template <int FT, typename TIn>
cudaError_t LaunchBaselinerT2(const BaselinerArgs& a, const KParams& k, cudaStream_t s)
{
    return a.map.On() ? LaunchBaselinerT3<FT, TIn, true>(a, k, s) : LaunchBaselinerT3<FT, TIn, false>(a, k, s);
}

template <int FT>
cudaError_t LaunchBaselinerT(const BaselinerArgs& a, const KParams& k, cudaStream_t s)
{
    const bool u8 = a.map.On() ? a.u8 != 0 : a.trace8 != nullptr;
    return u8 ? LaunchBaselinerT2<FT, uint8_t>(a, k, s) : LaunchBaselinerT2<FT, int16_t>(a, k, s);
}

cudaError_t LaunchBaseliner(int ft, const BaselinerArgs& a, const KParams& k, cudaStream_t s)
{
    switch (ft)
    {
    case 0: return LaunchBaselinerT<0>(a, k, s);
    case 1: return LaunchBaselinerT<1>(a, k, s);
    case 2: return LaunchBaselinerT<2>(a, k, s);
    case 3: return LaunchBaselinerT<3>(a, k, s);
    case 4: return LaunchBaselinerT<4>(a, k, s);
    case 5: return LaunchBaselinerT<5>(a, k, s);
    }
    return cudaErrorInvalidValue;
}

cudaError_t LaunchBaselinerInit(int ft, int16_t* st16, float* st32, int lanes, cudaStream_t s)
{
    const int threads = 128;
    const int blocks = (lanes * kLane + threads - 1) / threads;
    switch (ft)
    {
    case 0: BaselinerInitKernel<0><<<blocks, threads, 0, s>>>(st16, st32, lanes); break;
    case 1: BaselinerInitKernel<1><<<blocks, threads, 0, s>>>(st16, st32, lanes); break;
    case 2: BaselinerInitKernel<2><<<blocks, threads, 0, s>>>(st16, st32, lanes); break;
    case 3: BaselinerInitKernel<3><<<blocks, threads, 0, s>>>(st16, st32, lanes); break;
    case 4: BaselinerInitKernel<4><<<blocks, threads, 0, s>>>(st16, st32, lanes); break;
    case 5: BaselinerInitKernel<5><<<blocks, threads, 0, s>>>(st16, st32, lanes); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}   // namespace hwk
