// Multi-scale morphological baseliner for sm_100a.
//
// Restates TA/HostMultiScaleBaseliner.cpp:95-212, TA/TraceFilters.cpp:11-57,
// TA/BlockFilterStage.cpp:9-25 and DT/BaselinerStatAccumulator.cpp:39-53
// (TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes).
//
// Design: one thread per pair of neighbouring ZMWs streams its chunk frame by
// frame (see "Two ZMWs per thread" below for the packed arithmetic).  The reference
// runs every filter stage in place over the whole block; because each stage is
// causal (output m depends on inputs m-w..m-1) and chunk lengths are multiples
// of the aggregate stride, the same values come out of a per-frame pipeline in
// which scale i is fed at frames t with t % cumStride_i == 0.  The final stage
// produces block i's lower/upper envelope at frame i*aggStride, exactly when the
// subtraction of that block starts, so the trace is read from HBM once and the
// baselined trace written once, with coalesced 128-byte warp accesses.  The
// window arrays of stages up to 11 wide live in shared memory, wider ones in
// global memory, which leaves room for 14 one-lane blocks per SM (measured:
// 3.45 ms a 1M-ZMW chunk against 4.10 ms with 17-wide windows in shared
// memory at 12 blocks, 8.4 ms with every window in global memory).
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
    static constexpr int kSmemMaxWidth = 11;           // wider windows stay in global memory (L1/L2)
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

// ---- Two ZMWs per thread ----------------------------------------------------
// A thread owns the neighbouring ZMWs 2t and 2t + 1 of its lane: their int16
// values travel as one 32-bit pair (ZMW 2t in the low half), so the window
// filters run as packed 16-bit min/max (one instruction for both ZMWs) and
// every load and store of trace, output and state moves both.  The filter
// state keeps its [slot][zmw] int16 layout: a pair is just two neighbouring
// slots.  All ZMWs of a pool take the same frames, so the block counters of
// the window stages are one value per lane.  The floating-point estimate and
// statistics run as f32x2 pairs (see hw_device.cuh) or per ZMW with the
// reference's operation order.

__device__ __forceinline__ uint32_t MaxS16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("max.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t MinS16x2(uint32_t a, uint32_t b)
{
    uint32_t r;
    asm("min.s16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ int16_t Lo16(uint32_t p) { return (int16_t)(p & 0xffffu); }
__device__ __forceinline__ int16_t Hi16(uint32_t p) { return (int16_t)(p >> 16); }
__device__ __forceinline__ uint32_t Pack16(int16_t lo, int16_t hi) { return (uint32_t)(uint16_t)lo | ((uint32_t)(uint16_t)hi << 16); }

template <bool IsMax> __device__ __forceinline__ uint32_t Op2(uint32_t a, uint32_t b)
{
    return IsMax ? MaxS16x2(a, b) : MinS16x2(a, b);
}
template <bool IsMax> constexpr uint32_t Identity2() { return IsMax ? 0x80008000u : 0x7fff7fffu; }

// One van Herk/Gil-Werman window stage for a ZMW pair.  The output for each
// input is the extremum of the W previous inputs (TraceFilters.cpp:11-57 with
// the window state of WindowBuffer.h; the initial window holds W zeros).  The
// state is the suffix extrema S of the previous block of W inputs, the
// running extremum P of the current block and the current block's inputs B;
// the output at block position c is op(S[c], P).  `base` points at S[0] of
// this thread and `stride` separates consecutive array elements.
template <int W, bool IsMax>
__device__ __forceinline__ uint32_t StageStep2(uint32_t* base, int stride, uint32_t& P, int& counter, uint32_t x)
{
    uint32_t* S = base;
    uint32_t* B = base + W * stride;
    const int c = counter;
    const uint32_t y = Op2<IsMax>(S[c * stride], P);
    B[c * stride] = x;
    P = Op2<IsMax>(P, x);
    if (c + 1 == W)
    {
        // New suffix extrema of the completed block.
        uint32_t acc = x;
        S[(W - 1) * stride] = acc;
#pragma unroll 1
        for (int j = W - 2; j >= 0; --j)
        {
            acc = Op2<IsMax>(B[j * stride], acc);
            S[j * stride] = acc;
        }
        P = Identity2<IsMax>();
        counter = 0;
    }
    else
    {
        counter = c + 1;
    }
    return y;
}

// Global-memory window stage with S[counter] held in a register, loaded one
// call ahead of its use (S changes only when a block completes), so the
// stage never waits for memory on its critical path.  At a block's end the
// inputs are read in batches of 4 before the batch's results are stored.
template <int W, bool IsMax>
__device__ __forceinline__ uint32_t StageStepG2(uint32_t* base, int stride, uint32_t& P, int& counter,
                                                uint32_t& sNext, uint32_t x)
{
    uint32_t* S = base;
    uint32_t* B = base + W * stride;
    const int c = counter;
    const uint32_t y = Op2<IsMax>(sNext, P);
    B[c * stride] = x;
    P = Op2<IsMax>(P, x);
    if (c + 1 == W)
    {
        uint32_t acc = x;
        S[(W - 1) * stride] = acc;
        constexpr int kBatch = 4;
#pragma unroll 1
        for (int j0 = W - 2; j0 >= 0; j0 -= kBatch)
        {
            uint32_t b[kBatch];
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (j0 - q >= 0) b[q] = B[(j0 - q) * stride];
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (j0 - q >= 0)
                {
                    acc = Op2<IsMax>(b[q], acc);
                    S[(j0 - q) * stride] = acc;
                }
        }
        sNext = acc;      // S[0]
        P = Identity2<IsMax>();
        counter = 0;
    }
    else
    {
        counter = c + 1;
        sNext = S[(c + 1) * stride];
    }
    return y;
}

struct StageMem2
{
    uint32_t* smem;     // this thread's column in shared memory
    int sstride;        // blockDim.x
    uint32_t* gmem;     // this pair's column of the global-resident arrays
    int gstride;        // nZmw / 2
    uint32_t* sNext;    // per global stage: S[counter], loaded ahead
};

// Filter state of one thread: P of every stage (a ZMW pair) and the lane's
// block counters.
template <int FT> struct PairState
{
    uint32_t P[2 * FLayout<FT>::nStages];
    int c[2 * FLayout<FT>::nStages];
};

template <int FT, bool Upper, int K>
__device__ __forceinline__ uint32_t Stage2(const StageMem2& m, PairState<FT>& ps, uint32_t x)
{
    using Lay = FLayout<FT>;
    constexpr int W = Lay::Width(K);
    constexpr int off = Lay::Offset(Upper, K);
    constexpr int i = Lay::Idx(Upper, K);
    if constexpr (Lay::InSmem(K))
        return StageStep2<W, Lay::IsMax(Upper, K)>(m.smem + off * m.sstride, m.sstride, ps.P[i], ps.c[i], x);
    else
        return StageStepG2<W, Lay::IsMax(Upper, K)>(m.gmem + (size_t)off * m.gstride, m.gstride, ps.P[i], ps.c[i],
                                                    m.sNext[Lay::GIdx(Upper, K)], x);
}

// sNext of every global-memory stage of one filter from the saved state
// (compile-time recursion: the stage layout tables are host constants).
template <int FT, bool Upper, int K>
__device__ __forceinline__ void LoadSNext2(const StageMem2& m, const PairState<FT>& ps)
{
    using Lay = FLayout<FT>;
    if constexpr (K < Lay::nStages)
    {
        if constexpr (!Lay::InSmem(K))
        {
            constexpr int i = Lay::Idx(Upper, K);
            constexpr int off = Lay::Offset(Upper, K);
            m.sNext[Lay::GIdx(Upper, K)] = m.gmem[((size_t)off + (size_t)ps.c[i]) * (size_t)m.gstride];
        }
        LoadSNext2<FT, Upper, K + 1>(m, ps);
    }
}

template <int FT, bool Upper, int Scale>
__device__ __forceinline__ uint32_t RunScale2(const StageMem2& m, PairState<FT>& ps, uint32_t x)
{
    const uint32_t y = Stage2<FT, Upper, 2 * Scale>(m, ps, x);
    return Stage2<FT, Upper, 2 * Scale + 1>(m, ps, y);
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
__device__ __forceinline__ bool FeedFilter2(uint32_t x, const StageMem2& m, PairState<FT>& ps, uint32_t& out)
{
    using S = FSpec<FT>;
    using Lay = FLayout<FT>;
    static_assert(Lay::CumStride(0) <= 2 && (S::n < 2 || Lay::CumStride(1) <= 16) && Lay::AggStride() == 16,
                  "phase scheme needs cumulative strides 1|2, 2, 16");
    if constexpr (!ScaleRuns<Phase>(Lay::CumStride(0))) return false;
    uint32_t y = RunScale2<FT, Upper, 0>(m, ps, x);
    if constexpr (S::n > 1)
    {
        if constexpr (!ScaleRuns<Phase>(Lay::CumStride(1))) return false;
        y = RunScale2<FT, Upper, 1>(m, ps, y);
    }
    if constexpr (S::n > 2)
    {
        if constexpr (!ScaleRuns<Phase>(Lay::CumStride(2))) return false;
        y = RunScale2<FT, Upper, 2>(m, ps, y);
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

constexpr int kBlPairs = kLane / 2;       // threads per lane

// Reads the trace value pair of frame t.
template <typename TIn>
__device__ __forceinline__ uint32_t LoadPair(const TIn* tr, int t)
{
    if constexpr (std::is_same_v<TIn, uint8_t>)
    {
        const uint16_t b = __ldg(reinterpret_cast<const uint16_t*>(tr + (size_t)t * kLane));
        return (b & 0xffu) | ((uint32_t)(b >> 8) << 16);      // uint8 -> int16 widening of both
    }
    else
    {
        return __ldg(reinterpret_cast<const uint32_t*>(tr + (size_t)t * kLane));
    }
}

__device__ __forceinline__ float2 PairToFloat(uint32_t p) { return f2((float)Lo16(p), (float)Hi16(p)); }

// x - pedestal with int16 wrap-around, per half.
__device__ __forceinline__ uint32_t SubPed(uint32_t x, int16_t ped)
{
    return Pack16(i16_wrap(Lo16(x) - ped), i16_wrap(Hi16(x) - ped));
}

template <int FT, typename TIn, bool Mapped>
__global__ void __launch_bounds__(kBlPairs, 14) BaselinerKernel(BaselinerArgs a, KParams k)
{
    using Lay = FLayout<FT>;
    LaneMap map = a.map;
    if (!Mapped) map.list = nullptr;      // the single-pool variant compiles without the lane list
    // one lane per block, one ZMW pair per thread
    if ((int)blockIdx.x >= map.Lanes(a.lanes)) return;
    const int t = threadIdx.x;
    const int lane = map.Lane(blockIdx.x);
    const int nZmw = a.lanes * kLane;
    const int nPair = nZmw / 2;
    const int gp = lane * kBlPairs + t;       // pair index; ZMWs 2 gp, 2 gp + 1
    const int g = 2 * gp;
    const int z = 2 * t;
    const PoolStep* ps = map.On() ? &map.Pool(lane) : nullptr;
    const int F = ps ? ps->F : a.F;

    // Window state: narrow windows in shared memory (one column per thread),
    // wide ones used in place in global memory.
    extern __shared__ uint32_t blSmem2[];
    constexpr int SS = Lay::SmemSlots();
    constexpr int NG = Lay::NumGlobalStages() > 0 ? Lay::NumGlobalStages() : 1;
    uint32_t sNext[NG];
    const uint32_t* st = reinterpret_cast<const uint32_t*>(a.st16);
    uint32_t* stw = reinterpret_cast<uint32_t*>(a.st16);
    const StageMem2 mem{blSmem2 + t, kBlPairs, stw + (size_t)Lay::SlotGlobal() * nPair + gp, nPair, sNext};
#pragma unroll 32
    for (int i = 0; i < SS; ++i) blSmem2[i * kBlPairs + t] = st[(size_t)(Lay::SlotSmem() + i) * nPair + gp];
    PairState<FT> fs;
#pragma unroll
    for (int i = 0; i < 2 * Lay::nStages; ++i)
    {
        const bool up = i >= Lay::nStages;
        const int kk = up ? i - Lay::nStages : i;
        fs.P[i] = st[(size_t)Lay::SlotPC(up, kk) * nPair + gp];
        fs.c[i] = Lo16(st[(size_t)(Lay::SlotPC(up, kk) + 1) * nPair + gp]);   // the same for every ZMW
    }
    // S[counter] of every global stage
    LoadSNext2<FT, false, 0>(mem, fs);
    LoadSNext2<FT, true, 0>(mem, fs);
    uint32_t latData = st[(size_t)Lay::SlotLatData() * nPair + gp];
    uint32_t latRaw = st[(size_t)(Lay::SlotLatData() + 1) * nPair + gp];
    const uint32_t mbits = st[(size_t)(Lay::SlotLatData() + 2) * nPair + gp];
    bool latL0 = mbits & 1, latH10 = (mbits >> 1) & 1, latH20 = (mbits >> 2) & 1;
    bool latL1 = (mbits >> 16) & 1, latH11 = (mbits >> 17) & 1, latH21 = (mbits >> 18) & 1;
    const float2* st32 = reinterpret_cast<const float2*>(a.st32);
    float2 uemaSum = st32[(size_t)0 * nPair + gp];
    float2 uemaWeight = st32[(size_t)1 * nPair + gp];
    float2 sigmaEma = st32[(size_t)2 * nPair + gp];
    const float2 nz = f2(k.negZero);

    // Per-chunk BaselinerStatAccumulator (fresh each chunk, offset 0).  The
    // frame counts are the same for both ZMWs.
    float c_m0 = 0.0f;
    float2 c_m1 = f2(0.0f), c_m2 = f2(0.0f), c_acm2 = f2(0.0f);
    float2 fb0 = f2(0.0f), fb1 = f2(0.0f), fb2 = f2(0.0f), fb3 = f2(0.0f);
    float2 q0 = f2(0.0f), q1 = f2(0.0f), q2 = f2(0.0f), q3 = f2(0.0f);     // back buffer as a FIFO, q0 oldest
    int nAdded = 0;
    uint32_t tmin = 0x7fff7fffu, tmax = 0x80008000u;
    float2 b_m0 = f2(0.0f), b_m1 = f2(0.0f), b_m2 = f2(0.0f), rawSum = f2(0.0f);
    float g_m0 = 0.0f;
    float2 g_m1 = f2(0.0f), g_m2 = f2(0.0f);

    const TIn* tr;
    const size_t inOff = ps ? (size_t)(lane - ps->lane0) * F * kLane : (size_t)lane * F * kLane;
    if constexpr (std::is_same_v<TIn, uint8_t>) tr = (ps ? ps->trace8 : a.trace8) + inOff + z;
    else tr = (ps ? ps->trace : a.trace) + inOff + z;
    uint32_t* out = reinterpret_cast<uint32_t*>(a.out + map.Block(lane, F) + z);
    const int16_t ped = (int16_t)k.pedestal;
    const float2 scaler = f2(k.scaler);
    float2 sub = f2(0.0f);

    // Frames go in blocks of 16 (the aggregate stride): the first frame of a
    // block, the other even frames and the odd frames each get their own
    // specialisation of the frame body, with the trace loaded two frames ahead.
    // Even frames take their value from xEven and odd frames from xOdd, each
    // refilled right after use: no register is copied while its load is in
    // flight.
    static_assert(Lay::AggStride() == 16, "block size must be the aggregate stride");
    uint32_t xEven = LoadPair(tr, 0), xOdd = LoadPair(tr, 1);
    auto frame = [&](auto phaseTag, int f) {
        constexpr int Ph = decltype(phaseTag)::value;
        uint32_t& slot = (Ph == 2) ? xOdd : xEven;      // phase 2 = odd frames
        const uint32_t x = slot;
        if (f + 2 < F) slot = LoadPair(tr, f + 2);
        uint32_t lo = 0, up = 0;
        const bool haveL = FeedFilter2<FT, false, Ph>(x, mem, fs, lo);
        FeedFilter2<FT, true, Ph>(x, mem, fs, up);
        if (haveL)
        {
            // GetSmoothedBlEstimate (HostMultiScaleBaseliner.cpp:179-212)
            const uint32_t lv = SubPed(lo, ped), uv = SubPed(up, ped);
            constexpr float minSigma = .288675135f;
            const float ma = k.meanEmaAlpha, sa = k.sigmaEmaAlpha;
            float2 sigma;
            sigma.x = fmax_sse((float)i16_wrap(Lo16(uv) - Lo16(lv)) / k.cSigmaBias, minSigma);
            sigma.y = fmax_sse((float)i16_wrap(Hi16(uv) - Hi16(lv)) / k.cSigmaBias, minSigma);
            const float2 newSigmaEma = add2(mulz2(f2(sa), sigmaEma, nz), mulz2(f2(1.0f - sa), sigma, nz));
            const float2 mid = f2((float)i16_wrap(Lo16(uv) + Lo16(lv)), (float)i16_wrap(Hi16(uv) + Hi16(lv)));
            const float2 blEst = add2(mulz2(f2(0.5f), mid, nz), mulz2(f2(k.cMeanBias), newSigmaEma, nz));
            const float2 jt = mul2(f2(k.jumpTolCoeff), sigmaEma);
            const bool mx = (uemaWeight.x == 0.0f) | (blEst.x - uemaSum.x / uemaWeight.x < jt.x);
            const bool my = (uemaWeight.y == 0.0f) | (blEst.y - uemaSum.y / uemaWeight.y < jt.y);
            const float2 newWeight = add2(mulz2(f2(ma), uemaWeight, nz), f2(1.0f - ma));
            const float2 newSum = add2(mulz2(f2(ma), uemaSum, nz), mulz2(f2(1.0f - ma), blEst, nz));
            uemaWeight = f2(mx ? newWeight.x : uemaWeight.x, my ? newWeight.y : uemaWeight.y);
            uemaSum = f2(mx ? newSum.x : uemaSum.x, my ? newSum.y : uemaSum.y);
            sigmaEma = f2(mx ? newSigmaEma.x : sigmaEma.x, my ? newSigmaEma.y : sigmaEma.y);
            const float2 est = f2(uemaSum.x / uemaWeight.x, uemaSum.y / uemaWeight.y);
            sub = mulz2(est, scaler, nz);      // feeds the subtraction of every frame
            // AddSampleBackground (BaselinerStatAccumulator.cpp:56-60)
            const float2 bg = f2((float)to_i16_wrap(sub.x), (float)to_i16_wrap(sub.y));
            g_m0 += 1.0f;
            g_m1 = add2(g_m1, bg);
            g_m2 = add2(g_m2, mulz2(bg, bg, nz));
        }
        const uint32_t xp = SubPed(x, ped);
        const float2 rs = mulz2(PairToFloat(xp), scaler, nz);
        const float2 d = add2(rs, f2(-sub.x, -sub.y));
        const int16_t blsX = to_i16_wrap(d.x), blsY = to_i16_wrap(d.y);
        const uint32_t bls = Pack16(blsX, blsY);
        out[(size_t)f * (kLane / 2)] = bls;
        const uint32_t raw = Pack16(to_i16_wrap(rs.x), to_i16_wrap(rs.y));

        // AddToBaselineStats (HostMultiScaleBaseliner.cpp:148-176)
        const float2 thr = mul2(mul2(f2(4.5f), sigmaEma), scaler);
        const float2 fb = f2((float)blsX, (float)blsY);
        const bool hpX = fb.x < thr.x, hpY = fb.y < thr.y;
        const bool mX = latH10 & latL0 & hpX, mY = latH11 & latL1 & hpY;
        latL0 = hpX; latL1 = hpY;
        latH20 = latH10; latH21 = latH11;
        latH10 = hpX; latH11 = hpY;
        {
            // BaselinerStatAccumulator::AddSample(latRaw, latData, m)
            const float2 v = PairToFloat(latData);
            if (nAdded < 4)
            {
                if (nAdded == 0) fb0 = v; else if (nAdded == 1) fb1 = v; else if (nAdded == 2) fb2 = v; else fb3 = v;
            }
            c_acm2 = add2(c_acm2, mulz2(q0, v, nz));
            q0 = q1; q1 = q2; q2 = q3; q3 = v;
            ++nAdded;
            c_m0 += 1.0f;
            c_m1 = add2(c_m1, v);
            const float2 vv = mulz2(v, v, nz);
            c_m2 = add2(c_m2, vv);
            tmin = MinS16x2(latData, tmin);
            tmax = MaxS16x2(latData, tmax);
            const float2 a0 = add2(b_m0, f2(1.0f)), a1 = add2(b_m1, v), a2 = add2(b_m2, vv);
            b_m0 = f2(mX ? a0.x : b_m0.x, mY ? a0.y : b_m0.y);
            b_m1 = f2(mX ? a1.x : b_m1.x, mY ? a1.y : b_m1.y);
            b_m2 = f2(mX ? a2.x : b_m2.x, mY ? a2.y : b_m2.y);
            rawSum = add2(rawSum, f2((float)(mX ? Lo16(latRaw) : (int16_t)0), (float)(mY ? Hi16(latRaw) : (int16_t)0)));
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
    for (int i = 0; i < SS; ++i) stw[(size_t)(Lay::SlotSmem() + i) * nPair + gp] = blSmem2[i * kBlPairs + t];
#pragma unroll
    for (int i = 0; i < 2 * Lay::nStages; ++i)
    {
        const bool up = i >= Lay::nStages;
        const int kk = up ? i - Lay::nStages : i;
        stw[(size_t)Lay::SlotPC(up, kk) * nPair + gp] = fs.P[i];
        stw[(size_t)(Lay::SlotPC(up, kk) + 1) * nPair + gp] = Pack16((int16_t)fs.c[i], (int16_t)fs.c[i]);
    }
    stw[(size_t)Lay::SlotLatData() * nPair + gp] = latData;
    stw[(size_t)(Lay::SlotLatData() + 1) * nPair + gp] = latRaw;
    stw[(size_t)(Lay::SlotLatData() + 2) * nPair + gp] =
        Pack16((int16_t)((latL0 ? 1 : 0) | (latH10 ? 2 : 0) | (latH20 ? 4 : 0)),
               (int16_t)((latL1 ? 1 : 0) | (latH11 ? 2 : 0) | (latH21 ? 4 : 0)));
    float2* st32w = reinterpret_cast<float2*>(a.st32);
    st32w[(size_t)0 * nPair + gp] = uemaSum;
    st32w[(size_t)1 * nPair + gp] = uemaWeight;
    st32w[(size_t)2 * nPair + gp] = sigmaEma;

    // Per-chunk stats (GetState of the accumulator).
    hw_baseliner_stats& S = a.stats[lane];
    auto put = [&](float* arr, float2 v) { *reinterpret_cast<float2*>(arr + z) = v; };
    put(S.full_autocorr.basic_stats.offset, f2(0.0f));
    put(S.full_autocorr.basic_stats.moment0, f2(c_m0));
    put(S.full_autocorr.basic_stats.moment1, c_m1);
    put(S.full_autocorr.basic_stats.moment2, c_m2);
    put(S.full_autocorr.moment2, c_acm2);
    const int fbi = nAdded < 4 ? nAdded : 4;
    const int bbi = nAdded % 4;
    put(S.full_autocorr.fbuf[0], fb0); put(S.full_autocorr.fbuf[1], fb1);
    put(S.full_autocorr.fbuf[2], fb2); put(S.full_autocorr.fbuf[3], fb3);
    // bBuf[(bbi + j) % 4] holds the j-th oldest of the last four samples.
    const float2 qq[4] = {q0, q1, q2, q3};
#pragma unroll
    for (int j = 0; j < 4; ++j) put(S.full_autocorr.bbuf[(bbi + j) % 4], qq[j]);
    *reinterpret_cast<uint16_t*>(&S.full_autocorr.bidx[0][z]) = (uint16_t)(fbi | (fbi << 8));
    *reinterpret_cast<uint16_t*>(&S.full_autocorr.bidx[1][z]) = (uint16_t)(bbi | (bbi << 8));
    *reinterpret_cast<uint32_t*>(&S.trace_min[z]) = tmin;
    *reinterpret_cast<uint32_t*>(&S.trace_max[z]) = tmax;
    put(S.baseline_stats.offset, f2(0.0f));
    put(S.baseline_stats.moment0, b_m0);
    put(S.baseline_stats.moment1, b_m1);
    put(S.baseline_stats.moment2, b_m2);
    put(S.raw_baseline_sum, rawSum);
    put(S.background_stats.offset, f2(0.0f));
    put(S.background_stats.moment0, f2(g_m0));
    put(S.background_stats.moment1, g_m1);
    put(S.background_stats.moment2, g_m2);
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
    const int threads = kBlPairs;
    const size_t smem = sizeof(uint32_t) * FLayout<FT>::SmemSlots() * threads;
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
