// Frame labeler: ROI gating + 13-state subframe Viterbi for sm_100a.
//
// Restates TA/FrameLabelerHost.cpp:54-612, TA/SubframeScorer.h:152-318 and
// TA/RoiHost.h:75-249 (TA = src/basecaller/basecaller/traceAnalysis).
//
// One thread per ZMW.  Per chunk a thread
//   1. runs the ROI forward recursion over the 24 latent frames and the chunk,
//      keeping the 2-bit ROI codes packed 16 per word in local memory, then
//      the backward recursion (1 bit per frame);
//   2. runs the max-plus Viterbi over 24 latent + F-8 chunk frames + 16
//      look-ahead frames in fp32 with the reference's operation order and
//      tie rule (a later source state wins ties);
//   3. stores one 28-bit traceback word per frame: the arg-max source of each
//      destination row, coded in 4 bits for the 9-way rows (baseline and the
//      four pulse-up rows) and 1 bit for the 2-way rows (full and down);
//   4. back-propagates the normalised end-state probabilities 16 frames,
//      picks the anchor state and traces back F frames.
// Traceback words live in a global scratch laid out [lane][frame][zmw] so
// each warp writes and reads one 128-byte line per frame.
#include "pulse_seg.cuh"

namespace hwk {

// BlockStateSubframeScorer for one ZMW (SubframeScorer.h:152-318).  The
// scores of analogs 0/1 and 2/3 are evaluated as packed pairs with the
// reference's operation order (see the f32x2 helpers); constants the
// reference recomputes per frame from per-ZMW values (-0.5 times the inverse
// variances, the negated caps, means and log means, the dimmest analog's
// fallback condition) are formed once in Setup, with the same roundings.
struct ZScorer
{
    float bgMean, bInvVar, bgFixed, x0, nhBInv;
    float2 negMean[2], pInv[2], ffFixed[2], nhPInv[2], negX1[2], negLogP[2], x1[2];
    float fbMean, fbNormTerm, fbScale;
    bool fbUse;     // x0 > x1 of the dimmest analog: its up/down score is the normal fallback

    __device__ __forceinline__ void Setup(const KParams& k, const hw_lane_model& m, int z)
    {
        constexpr float log2pi_f = 1.8378770664f;
        const float nhalf = -0.5f, halfVal = 0.5f, oneSixth = 1.0f / 6.0f;
        const float bMean = h2f(m.baseline.means[z]);
        const float bVar = h2f(m.baseline.vars[z]);
        const float bSigma = sqrtf(bVar);
        x0 = add_rn(bMean, mul_rn(bSigma, k.sqrtHalfPi));
        bInvVar = 1.0f / bVar;
        nhBInv = mul_rn(nhalf, bInvVar);
        float aM[kAnalogs], pI[kAnalogs], fx[kAnalogs], lp[kAnalogs], xx[kAnalogs];
#pragma unroll
        for (int a = 0; a < kAnalogs; ++a)
        {
            const float aMean = h2f(m.analogs[a].means[z]);
            lp[a] = hw_logf(aMean - bMean);
            const float aVar = h2f(m.analogs[a].vars[z]);
            const float aSigma = sqrtf(aVar);
            xx[a] = aMean - mul_rn(aSigma, k.sqrtHalfPi);
            pI[a] = 1.0f / aVar;
            fx[a] = mul_rn(nhalf, hw_logf(aVar)) - log2pi_f / 2.0f;
            aM[a] = aMean;
        }
#pragma unroll
        for (int q = 0; q < 2; ++q)
        {
            const int a = 2 * q;
            negMean[q] = f2(-aM[a], -aM[a + 1]);
            pInv[q] = f2(pI[a], pI[a + 1]);
            ffFixed[q] = f2(fx[a], fx[a + 1]);
            nhPInv[q] = f2(mul_rn(nhalf, pI[a]), mul_rn(nhalf, pI[a + 1]));
            negX1[q] = f2(-xx[a], -xx[a + 1]);
            x1[q] = f2(xx[a], xx[a + 1]);
            negLogP[q] = f2(-lp[a], -lp[a + 1]);
        }
        {
            const float aMean = aM[3];
            const float aVar = h2f(m.analogs[3].vars[z]);
            const float eMean = mul_rn(halfVal, bMean + aMean);
            float eVar = mul_rn(oneSixth, aMean - bMean);
            eVar = add_rn(eVar, bVar + aVar);
            eVar = mul_rn(eVar, halfVal);
            fbMean = eMean;
            fbNormTerm = mul_rn(-0.5f, add_rn(log2pi_f, hw_logf(eVar)));
            fbScale = 0.5f / eVar;
        }
        fbUse = !(x0 <= xx[3]);
        bgFixed = mul_rn(nhalf, hw_logf(bVar)) - log2pi_f / 2.0f;
        bgMean = bMean;
    }

    // StateScores for states 0..8 (states 9..12 repeat 5..8).
    __device__ __forceinline__ void Scores(float data, float* out, float2 nz) const
    {
        {
            const float y = data - bgMean;
            out[0] = add_rn(mul_rn(mul_rn(mul_rn(-0.5f, y), bInvVar), y), bgFixed);
        }
        const float2 d2 = f2(data);
        const bool low = data < x0;
#pragma unroll
        for (int q = 0; q < 2; ++q)
        {
            // full frame: ((-0.5 y) / var) y + fixed, y = data - mean
            const float2 y = add2(d2, negMean[q]);
            const float2 full = add2(mulz2(mul2(mul2(f2(-0.5f), y), pInv[q]), y, nz), ffFixed[q]);
            // sub-frame Gauss cap: (extrema ? (-0.5 / var) dv^2 : 0) - log(mean - baseline mean)
            const float2 negCap = low ? f2(-x0) : negX1[q];
            const float2 fixedTerm = low ? f2(nhBInv) : nhPInv[q];
            const float2 dv = add2(d2, negCap);
            const float2 prod = mulz2(fixedTerm, mul2(dv, dv), nz);
            const bool ex = low | (data > x1[q].x), ey = low | (data > x1[q].y);
            float2 sub = add2(f2(ex ? prod.x : 0.0f, ey ? prod.y : 0.0f), negLogP[q]);
            if (q == 1 && fbUse)
            {
                const float dm = data - fbMean;
                sub.y = fbNormTerm - mul_rn(mul_rn(dm, dm), fbScale);
            }
            // clamp above the full-frame mean
            const float2 fm1 = add2(full, f2(-1.0f));
            sub.x = (data > -negMean[q].x) ? fmin_sse(fmin_sse(sub.x, fm1.x), 0.0f) : sub.x;
            sub.y = (data > -negMean[q].y) ? fmin_sse(fmin_sse(sub.y, fm1.y), 0.0f) : sub.y;
            out[1 + 2 * q] = full.x;
            out[2 + 2 * q] = full.y;
            out[5 + 2 * q] = sub.x;
            out[6 + 2 * q] = sub.y;
        }
    }
};

// Log-likelihoods of the 13 states between Viterbi steps: state 0 alone,
// states 1..12 in the pairs (1,2) (3,4) (5,6) (7,8) (9,10) (11,12) that the
// rows add as one f32x2 operation (every row reads its sources pairwise:
// the 9-way rows (5,6) .. (11,12), the 2-way rows of states r and r + 1 read
// (r, r + 1) and (r + 4, r + 5) or (r - 8, r - 7) and (r - 4, r - 3)).
struct StateLL
{
    float s0;
    float2 p[6];
    __device__ __forceinline__ float Get(int i) const
    {
        return i == 0 ? s0 : (((i - 1) & 1) ? p[(i - 1) >> 1].y : p[(i - 1) >> 1].x);
    }
    __device__ __forceinline__ void Set(int i, float v)
    {
        if (i == 0) s0 = v;
        else if ((i - 1) & 1) p[(i - 1) >> 1].y = v;
        else p[(i - 1) >> 1].x = v;
    }
};

// Arg-max over a row's candidates in the reference's order (first entry,
// then the contiguous segment); ties go to the later entry (Recursion,
// FrameLabelerHost.cpp:214-264).  The candidate values are
// (score + T[row][src]) + ll[src]: the first addition per candidate, the
// second pairwise.  Instead of the source state a row returns its traceback
// code already shifted into place: 9-way rows (baseline, pulse-up) code
// source s as 0 for state 0 and s - 4 for states 5..12 in 4 bits; 2-way
// rows (full, down) code the second source as one bit, the outcome of their
// single comparison.  With Margin, `gap` receives the row's decision gap:
// the winning candidate less the best other one (0 on a tie, +inf when only
// one is finite).
template <bool Margin>
__device__ __forceinline__ void Pick(float v, uint32_t cv, float& mv, float& sv, uint32_t& c)
{
    const bool ge = v >= mv;
    if constexpr (Margin) sv = ge ? mv : ((v > sv) ? v : sv);
    mv = ge ? v : mv;
    c = ge ? cv : c;
}

template <int R, bool Margin>
__device__ __forceinline__ float NineWayRow(const KParams& k, float score, const StateLL& ll, uint32_t& code,
                                            float& gap)
{
    constexpr int shift = (R == 0) ? 0 : 4 + 4 * (R - 5);
    float mv = add_rn(add_rn(score, k.trans[R][0]), ll.s0);
    float sv = -__int_as_float(0x7f800000);
    uint32_t c = 0u;
#pragma unroll
    for (int q = 2; q < 6; ++q)
    {
        const int p0 = 2 * q + 1;          // sources p0, p0 + 1
        const float2 v = add2(add2(f2(score), f2(k.trans[R][p0], k.trans[R][p0 + 1])), ll.p[q]);
        Pick<Margin>(v.x, (uint32_t)(p0 - 4) << shift, mv, sv, c);
        Pick<Margin>(v.y, (uint32_t)(p0 - 3) << shift, mv, sv, c);
    }
    code = c;
    if constexpr (Margin) gap = mv - sv;
    return mv;
}

// Grouped 9-way rows.  When a row's transition constants are equal within
// each source group (t_A for states 5..8, t_B for 9..12; KParams::grouped9),
// its candidates of group G are RN(a_G + ll[s]) with a_G = RN(score + t_G)
// the same for the whole group, and RN(a_G + x) is monotone in x.  So the
// group's best value is RN(a_G + m_G), m_G the group's largest ll, reached
// by the last state holding m_G, unless a later state of the group rounds
// to the same sum: that needs RN(a_G + m'_G) == RN(a_G + m_G), m'_G the
// largest ll after that state, and sends the frame to the generic rows.  m_G,
// its last position and m'_G are shared by the five 9-way rows of a frame.
struct GroupMax
{
    float m;        // largest ll of the group
    float after;    // largest ll after its last position (NaN: none)
    uint32_t pos;   // last position of m, 0..3
};

// Right to left with strict comparisons: the last position of the maximum.
__device__ __forceinline__ GroupMax ScanGroup(float2 lo, float2 hi)
{
    GroupMax g{hi.y, __int_as_float(0x7fffffff), 3u};
    auto step = [&](float v, uint32_t p) {
        const bool gt = v > g.m;
        g.after = gt ? g.m : g.after;
        g.m = gt ? v : g.m;
        g.pos = gt ? p : g.pos;
    };
    step(hi.x, 2u);
    step(lo.y, 1u);
    step(lo.x, 0u);
    return g;
}

// One grouped 9-way row (index i of rows 0, 5, 6, 7, 8): returns the row's
// value; base receives the winner's code (0 for state 0, s - 4 for s in
// 5..12) unshifted; slow is set when the group winner is not certain.
template <int i>
__device__ __forceinline__ float GroupedRow(const KParams& k, float score, float ll0, float2 gm, float2 gafter,
                                            uint32_t codeA, uint32_t codeB, uint32_t& base, bool& slow)
{
    constexpr int R = (i == 0) ? 0 : i + 4;
    const float c0 = add_rn(add_rn(score, k.trans[R][0]), ll0);
    const float2 a = add2(f2(score), k.grp9[i]);
    const float2 gv = add2(a, gm);          // the groups' best candidates
    const float2 nv = add2(a, gafter);      // the best after each group's winner
    const bool geA = gv.x >= c0;
    const float mv = geA ? gv.x : c0;
    const bool geB = gv.y >= mv;
    base = geB ? codeB : (geA ? codeA : 0u);
    slow |= geB ? (nv.y == gv.y) : (geA & (nv.x == gv.x));
    return geB ? gv.y : mv;
}

// Two 2-way rows, R and R + 1, with scores s.x, s.y: their first sources are
// the pair qa, their second the pair qb.
template <int R, int qa, int qb, bool Margin>
__device__ __forceinline__ float2 TwoWayRows(const KParams& k, float2 s, const StateLL& ll, uint32_t& code,
                                             float& gap0, float& gap1)
{
    constexpr int shift = (R <= 4) ? 20 + R - 1 : 24 + R - 9;
    constexpr int a0 = 2 * qa + 1, b0 = 2 * qb + 1;
    const float2 first = add2(add2(s, f2(k.trans[R][a0], k.trans[R + 1][a0 + 1])), ll.p[qa]);
    const float2 second = add2(add2(s, f2(k.trans[R][b0], k.trans[R + 1][b0 + 1])), ll.p[qb]);
    const bool gx = second.x >= first.x, gy = second.y >= first.y;
    if constexpr (Margin)
    {
        const float ninf = -__int_as_float(0x7f800000);
        const float sx = gx ? first.x : ((second.x > ninf) ? second.x : ninf);
        const float sy = gy ? first.y : ((second.y > ninf) ? second.y : ninf);
        gap0 = (gx ? second.x : first.x) - sx;
        gap1 = (gy ? second.y : first.y) - sy;
    }
    code = (gx ? 1u << shift : 0u) | (gy ? 2u << shift : 0u);
    return f2(gx ? second.x : first.x, gy ? second.y : first.y);
}

// One Viterbi recursion step; returns the packed traceback word.  With
// Margin, gap[r] receives row r's decision gap.
template <bool Margin = false, bool Grouped = false>
__device__ __forceinline__ uint32_t ViterbiStep(const KParams& k, const ZScorer& sc, float data, bool isRoi,
                                                StateLL& ll, float* gap = nullptr)
{
    static_assert(!(Margin && Grouped), "margins come from the generic rows");
    float sco[9];
    sc.Scores(data, sco, f2(k.negZero));
    uint32_t cd[9];
    float gl[kStates];
    float n0, n5, n6, n7, n8;
    if constexpr (Grouped)
    {
        const GroupMax gA = ScanGroup(ll.p[2], ll.p[3]), gB = ScanGroup(ll.p[4], ll.p[5]);
        const float2 gm = f2(gA.m, gB.m), ga = f2(gA.after, gB.after);
        const uint32_t codeA = 1u + gA.pos, codeB = 5u + gB.pos;
        // a NaN among the rows' inputs (or an inf - inf) takes the generic rows
        const float2 lsum = add2(add2(ll.p[2], ll.p[3]), add2(ll.p[4], ll.p[5]));
        const float ssum = add_rn(add_rn(add_rn(sco[0], sco[5]), add_rn(sco[6], sco[7])), sco[8]);
        bool slow = isnan(add_rn(add_rn(lsum.x, lsum.y), add_rn(ll.s0, ssum)));
        uint32_t b0, b5, b6, b7, b8;
        n0 = GroupedRow<0>(k, sco[0], ll.s0, gm, ga, codeA, codeB, b0, slow);
        n5 = GroupedRow<1>(k, sco[5], ll.s0, gm, ga, codeA, codeB, b5, slow);
        n6 = GroupedRow<2>(k, sco[6], ll.s0, gm, ga, codeA, codeB, b6, slow);
        n7 = GroupedRow<3>(k, sco[7], ll.s0, gm, ga, codeA, codeB, b7, slow);
        n8 = GroupedRow<4>(k, sco[8], ll.s0, gm, ga, codeA, codeB, b8, slow);
        if (slow)
        {
            n0 = NineWayRow<0, false>(k, sco[0], ll, cd[0], gl[0]);
            n5 = NineWayRow<5, false>(k, sco[5], ll, cd[1], gl[5]);
            n6 = NineWayRow<6, false>(k, sco[6], ll, cd[2], gl[6]);
            n7 = NineWayRow<7, false>(k, sco[7], ll, cd[3], gl[7]);
            n8 = NineWayRow<8, false>(k, sco[8], ll, cd[4], gl[8]);
        }
        else
        {
            cd[0] = b0;
            cd[1] = b5 << 4;
            cd[2] = b6 << 8;
            cd[3] = b7 << 12;
            cd[4] = b8 << 16;
        }
    }
    else
    {
        n0 = NineWayRow<0, Margin>(k, sco[0], ll, cd[0], gl[0]);
        n5 = NineWayRow<5, Margin>(k, sco[5], ll, cd[1], gl[5]);
        n6 = NineWayRow<6, Margin>(k, sco[6], ll, cd[2], gl[6]);
        n7 = NineWayRow<7, Margin>(k, sco[7], ll, cd[3], gl[7]);
        n8 = NineWayRow<8, Margin>(k, sco[8], ll, cd[4], gl[8]);
    }
    // full rows: (r, r + 4); down rows: (r - 8, r - 4)
    const float2 n12 = TwoWayRows<1, 0, 2, Margin>(k, f2(sco[1], sco[2]), ll, cd[5], gl[1], gl[2]);
    const float2 n34 = TwoWayRows<3, 1, 3, Margin>(k, f2(sco[3], sco[4]), ll, cd[6], gl[3], gl[4]);
    const float2 n9a = TwoWayRows<9, 0, 2, Margin>(k, f2(sco[5], sco[6]), ll, cd[7], gl[9], gl[10]);
    const float2 nbc = TwoWayRows<11, 1, 3, Margin>(k, f2(sco[7], sco[8]), ll, cd[8], gl[11], gl[12]);
    // non-ROI frames: every state but the baseline gets -inf (x - inf)
    const float2 npen = f2(isRoi ? -0.0f : -__int_as_float(0x7f800000));
    ll.s0 = n0;
    ll.p[0] = add2(n12, npen);
    ll.p[1] = add2(n34, npen);
    ll.p[2] = add2(f2(n5, n6), npen);
    ll.p[3] = add2(f2(n7, n8), npen);
    ll.p[4] = add2(n9a, npen);
    ll.p[5] = add2(nbc, npen);
    if constexpr (Margin)
    {
#pragma unroll
        for (int r = 0; r < kStates; ++r) gap[r] = gl[r];
    }
    return ((cd[0] | cd[1] | cd[2]) | (cd[3] | cd[4])) | ((cd[5] | cd[6]) | (cd[7] | cd[8]));
}

// Source state of `state` recorded in traceback word `w`.
__device__ __forceinline__ int TraceSource(uint32_t w, int state)
{
    if (state == 0 || state >= 5 && state <= 8)
    {
        const int shift = (state == 0) ? 0 : 4 + 4 * (state - 5);
        const int c = (w >> shift) & 15u;
        return c == 0 ? 0 : c + 4;
    }
    if (state <= 4)
    {
        const int b = (w >> (20 + state - 1)) & 1u;
        return b ? state + 4 : state;
    }
    const int b = (w >> (24 + state - 9)) & 1u;
    return b ? state - 4 : state - 8;
}


// x / c, correctly rounded, for the ROI's constants c = sqrt(2) and sqrt(3):
// q = x * RN(1/c) corrected once with the exact remainder x - q c (Markstein's
// correction); zero and non-finite quotients pass through.  An exhaustive
// check over every float x gives the IEEE quotient for both constants
// whenever |x| >= 2^-100 (the largest x that differs is below 2^-102), and
// for zero, infinite and NaN x; only smaller x can differ, and the ROI never
// divides one (its dividends are 0 or sums of int16 trace values times an
// inverse sigma of at least 1/256, so their magnitude is 0 or above 2^-33).
__device__ __forceinline__ float DivByConst(float x, float c, float rcp)
{
    const float q = mul_rn(x, rcp);
    const float r = fma_rn(-q, c, x);
    const float q2 = fma_rn(r, rcp, q);
    return (isfinite(q) && q != 0.0f) ? q2 : q;
}

constexpr int kBatch = 8;                              // frames loaded ahead

// L1 prefetch of one address, no register result: used where the next loads
// are needed sooner than one loop iteration can hide (the ROI pass spends ~30
// instructions a frame) and for the traceback words read back in batches.
__device__ __forceinline__ void PrefetchL1(const void* p) { asm volatile("prefetch.global.L1 [%0];" :: "l"(p)); }


// Blocks per SM the labeler variants are compiled for (96 registers a thread).
constexpr int LabelerMinBlocks(int threads) { return threads == 64 ? 10 : threads == 128 ? 5 : 2; }

// Mapped: lane-list launch.  Fuse: the pulse accumulator runs in the same
// thread right after the traceback, on labels kept in shared memory (4 bits a
// frame) instead of a labels batch in global memory.  Threads: 64 ZMWs (one
// lane) per 64 threads.
// Margin (single-pool launch only): the decision gaps of every frame and
// state go to the scratch A.gap [lanes][F + 16][13][64], and the traceback
// writes each label's best-path margin to A.margin.
template <bool Mapped, bool Fuse, int Threads, bool Margin = false, bool Grouped = false>
__global__ void __launch_bounds__(Threads, LabelerMinBlocks(Threads)) LabelerKernel(LabelerArgs A, KParams k,
                                                                                     PulseArgs P)
{
    static_assert(!Margin || (!Mapped && !Fuse), "margins come from the single-pool labeler");
    static_assert(!(Margin && Grouped), "margins come from the generic rows");
    LaneMap map = A.map;
    if (!Mapped) map.list = nullptr;      // the single-pool variant compiles without the lane list
    int l, z;
    if (!ZmwOf(map, A.lanes, l, z)) return;
    const int g = l * kLane + z;
    const int F = map.On() ? map.Pool(l).F : A.F;
    const int nRoi = F + kLookback + kStitch;
    const int16_t* chunk = A.trace + map.Block(l, F) + z;
    int16_t* pl = A.prevLat + (size_t)l * kLatent * kLane + z;
    const hw_lane_model& oldM = A.latModel[l];
    const hw_lane_model& newM = A.models[l];

    // ---- ROI (ComputeRoi, FrameLabelerHost.cpp:267-309; RoiHost.h:110-249)
    // 2-bit ROI codes, 16 per word, in dynamic shared memory [word][thread]
    // (kept out of local memory, whose L1 share depends on other kernels'
    // shared-memory carve-out).
    extern __shared__ uint32_t roiSh[];
    auto roiw = [&](int w) -> uint32_t& { return roiSh[w * blockDim.x + threadIdx.x]; };
    {
        const float inv1 = 1.0f / sqrtf(h2f(oldM.baseline.vars[z]));
        const float inv2 = 1.0f / sqrtf(h2f(newM.baseline.vars[z]));
        float p0 = mul_rn((float)A.latTrc[g], inv1);
        float p1 = mul_rn((float)pl[0], inv1);
        float p2 = mul_rn((float)pl[kLane], inv1);
        uint32_t prevRoi = (uint16_t)A.latRoi[g];
        uint32_t word = 0;
        int ri = 0;
        auto process = [&](float sn) {
            float mval = p1;
            mval = fmax_sse(mval, DivByConst(p0 + p1, k.sqrt2, k.rcpSqrt2));
            mval = fmax_sse(mval, DivByConst(add_rn(p0 + p1, p2), k.sqrt3, k.rcpSqrt3));
            mval = fmax_sse(mval, add_rn(add_rn(p0 + p1, p2), sn) / 2.0f);
            const float thresh = (prevRoi & 1u) ? k.roiLower : k.roiUpper;
            const uint32_t v = ((mval >= thresh) ? 1u : 0u) | ((mval >= k.roiLower) ? 2u : 0u);
            word |= v << (2 * (ri & 15));
            if ((ri & 15) == 15) { roiw(ri >> 4) = word; word = 0; }
            ++ri;
            prevRoi = v;
            p0 = p1; p1 = p2; p2 = sn;
        };
        for (int i = hwp::kRoiLookForward; i < kLatent; ++i) process(mul_rn((float)pl[(size_t)i * kLane], inv1));
        {
            int16_t y0 = __ldg(chunk), y1 = __ldg(chunk + kLane);
#pragma unroll 2
            for (int i = 0; i < F; ++i)
            {
                if (i + 8 < F) PrefetchL1(chunk + (size_t)(i + 8) * kLane);
                const int16_t y = y0;
                y0 = y1;
                if (i + 2 < F) y1 = __ldg(chunk + (size_t)(i + 2) * kLane);
                process(mul_rn((float)y, inv2));
            }
        }
        if (ri & 15) roiw(ri >> 4) = word;
        // Backward recursion: 2-bit codes become 0/1 (in place, bit 0 of each code).
        uint32_t pr = 0;
        for (int wi = (nRoi - 1) >> 4; wi >= 0; --wi)
        {
            uint32_t wv = roiw(wi);
            uint32_t outw = 0;
            const int hi = (wi == ((nRoi - 1) >> 4)) ? ((nRoi - 1) & 15) : 15;
            for (int j = hi; j >= 0; --j)
            {
                const uint32_t code = (wv >> (2 * j)) & 3u;
                const uint32_t b = (code & 1u) | (((code & 2u) != 0u) & (pr != 0u));
                pr = b;
                outw |= b << (2 * j);
            }
            roiw(wi) = outw;
        }
    }
    auto roiBit = [&](int f) -> bool { return (roiw(f >> 4) >> (2 * (f & 15))) & 1u; };

    // ---- Viterbi (LabelBlock, FrameLabelerHost.cpp:314-448)
    StateLL ll;
    {
        const int bc = A.latLabel[g];
#pragma unroll
        for (int i = 0; i < kStates; ++i) ll.Set(i, (bc == i) ? 0.0f : -__int_as_float(0x7f800000));
    }
    uint32_t* tb = A.tb + map.BlockX(l, F, kLookback) + z;
    // decision gap of state r at frame lf
    auto gapAt = [&](int lf, int r) -> float& {
        return A.gap[(((size_t)l * (F + kLookback) + lf) * kStates + r) * kLane + z];
    };
    ZScorer sc;
    auto step = [&](int lf, float x, bool isRoi) {
        if constexpr (Margin)
        {
            float g[kStates];
            tb[(size_t)lf * kLane] = ViterbiStep<true>(k, sc, x, isRoi, ll, g);
#pragma unroll
            for (int r = 0; r < kStates; ++r) gapAt(lf, r) = g[r];
        }
        else
        {
            tb[(size_t)lf * kLane] = ViterbiStep<false, Grouped>(k, sc, x, isRoi, ll);
        }
    };
    sc.Setup(k, oldM, z);
    uint32_t roiWord = roiw(0);
    for (int f = 0; f < kLatent; ++f)
    {
        if ((f & 15) == 0) roiWord = roiw(f >> 4);
        const bool isRoi = (roiWord >> (2 * (f & 15))) & 1u;
        step(f, (float)pl[(size_t)f * kLane], isRoi);
    }
    sc.Setup(k, newM, z);
    const int anchor = F - kLatent;
    float anchorLL[kStates];
    // Chunk frames 0 .. anchor + 15 (labels kLatent .. F + 15).  The loop
    // stays rolled (one Viterbi step is several hundred instructions; copies
    // of it overflow the instruction cache) and the trace is loaded two
    // frames ahead of use.
    const int nFrames = anchor + kLookback;
    int16_t x0 = __ldg(chunk), x1 = __ldg(chunk + kLane);
#pragma unroll 1
    for (int f = 0; f < nFrames; ++f)
    {
        const int16_t x = x0;
        x0 = x1;
        if (f + 2 < nFrames) x1 = __ldg(chunk + (size_t)(f + 2) * kLane);
        if (f == anchor)
        {
#pragma unroll
            for (int i = 0; i < kStates; ++i) anchorLL[i] = ll.Get(i);
        }
        const int lf = f + kLatent;
        if ((lf & 15) == 0) roiWord = roiw(lf >> 4);
        const bool isRoi = (roiWord >> (2 * (lf & 15))) & 1u;
        step(lf, (float)x, isRoi);
    }

    // Normalize (FrameLabelerHost.cpp:186-205) and back-propagation.
    float prob[kStates];
    {
        float mx = ll.Get(0);
#pragma unroll
        for (int i = 1; i < kStates; ++i) mx = fmax_sse(ll.Get(i), mx);
        float sum = 0.0f;
#pragma unroll
        for (int i = 0; i < kStates; ++i) { prob[i] = hw_expf(ll.Get(i) - mx); sum = add_rn(sum, prob[i]); }
        const float inv = 1.0f / sum;
#pragma unroll
        for (int i = 0; i < kStates; ++i) prob[i] = mul_rn(prob[i], inv);
    }
    for (int i = F + kLookback - 1; i > F - 1; --i) PrefetchL1(tb + (size_t)i * kLane);
    for (int i = F + kLookback - 1; i > F - 1; --i)
    {
        const uint32_t w = tb[(size_t)i * kLane];
        float np[kStates];
#pragma unroll
        for (int s = 0; s < kStates; ++s) np[s] = 0.0f;
#pragma unroll
        for (int from = 0; from < kStates; ++from)
        {
            const int to = TraceSource(w, from);
#pragma unroll
            for (int s = 0; s < kStates; ++s) np[s] = (s == to) ? add_rn(np[s], prob[from]) : np[s];
        }
#pragma unroll
        for (int s = 0; s < kStates; ++s) prob[s] = np[s];
    }
    float maxP = prob[0];
    int anchorState = 0;
#pragma unroll
    for (int i = 1; i < kStates; ++i)
    {
        const bool c = maxP > prob[i];
        maxP = c ? maxP : prob[i];
        anchorState = c ? anchorState : i;
    }
    float ret = anchorLL[0];
#pragma unroll
    for (int i = 1; i < kStates; ++i) ret = (anchorState == i) ? anchorLL[i] : ret;

    int ts = anchorState;
    if constexpr (Fuse)
    {
        // The ROI words are done with: the last ROI bit goes to the latent
        // state first, then the traceback packs 8 labels a word into them.
        A.latRoi[g] = (int16_t)roiBit(F - 1);
        for (int f0 = F - kBatch; f0 >= 0; f0 -= kBatch)
        {
            uint32_t w[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; ++j) w[j] = tb[(size_t)(f0 + j) * kLane];
            if (f0 >= kBatch)
            {
#pragma unroll
                for (int j = 0; j < kBatch; ++j) PrefetchL1(tb + (size_t)(f0 - kBatch + j) * kLane);
            }
            uint32_t word = 0;
#pragma unroll
            for (int j = kBatch - 1; j >= 0; --j)
            {
                word |= (uint32_t)ts << (4 * j);
                ts = TraceSource(w[j], ts);
            }
            roiw(f0 / kBatch) = word;
        }
        // Pulse accumulation over the labels batch (frames chunk start - 24
        // .. chunk end - 24): the previous chunk's latent frames, then the
        // chunk's first F - 24 frames.
        const PoolStep& ps = map.Pool(l);
        const int go = (l - ps.lane0) * kLane + z;
        const uint32_t firstFrame = (uint32_t)(ps.firstFrame - kLatent);
        PulseSeg seg;
        seg.Load(P, g, h2f(newM.analogs[kAnalogs - 1].means[z]), ps.pulses + (size_t)go * k.maxCalls);
        for (int r0 = 0; r0 < F; r0 += kBatch)
        {
            const uint32_t word = roiw(r0 / kBatch);
            int16_t sg[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; ++j)
            {
                const int r = r0 + j;
                sg[j] = (r < kLatent) ? pl[(size_t)r * kLane] : __ldg(chunk + (size_t)(r - kLatent) * kLane);
            }
#pragma unroll
            for (int j = 0; j < kBatch; ++j)
                seg.Frame(k, (uint32_t)(r0 + j) + firstFrame, (int16_t)((word >> (4 * j)) & 15u), sg[j]);
            seg.Flush(k);
        }
        seg.Store(P, g, l, z, ps.lens, ps.ovf, go);
    }
    else if constexpr (Margin)
    {
        // Traceback with the best path's decision margin of every label: the
        // last label's is the anchor choice's probability gap, label f's the
        // gap that frame f + 1 recorded for the path's state there.
        int16_t* out = A.labels + map.Block(l, F) + z;
        float* mg = A.margin + map.Block(l, F) + z;
        float second = -__int_as_float(0x7f800000);
#pragma unroll
        for (int i = 0; i < kStates; ++i) second = (i != anchorState && prob[i] > second) ? prob[i] : second;
        mg[(size_t)(F - 1) * kLane] = maxP - second;
        int next = anchorState;
        for (int f = F - 1; f >= 0; --f)
        {
            out[(size_t)f * kLane] = (int16_t)ts;
            if (f < F - 1) mg[(size_t)f * kLane] = gapAt(f + 1, next);
            next = ts;
            ts = TraceSource(tb[(size_t)f * kLane], ts);
        }
        A.latRoi[g] = (int16_t)roiBit(F - 1);
    }
    else
    {
        // the labels block sits at the chunk's offset (derived from the
        // chunk pointer, so the lane map need not stay live through the loop)
        int16_t* out = A.labels + (chunk - A.trace);
        for (int f0 = F - kBatch; f0 >= 0; f0 -= kBatch)
        {
            uint32_t w[kBatch];
#pragma unroll
            for (int j = 0; j < kBatch; ++j) w[j] = tb[(size_t)(f0 + j) * kLane];
            if (f0 >= kBatch)
            {
#pragma unroll
                for (int j = 0; j < kBatch; ++j) PrefetchL1(tb + (size_t)(f0 - kBatch + j) * kLane);
            }
#pragma unroll
            for (int j = kBatch - 1; j >= 0; --j)
            {
                out[(size_t)(f0 + j) * kLane] = (int16_t)ts;
                ts = TraceSource(w[j], ts);
            }
        }
        A.latRoi[g] = (int16_t)roiBit(F - 1);
    }

    // Latent state update.
    A.latLabel[g] = (int16_t)anchorState;
    A.latTrc[g] = chunk[(size_t)(anchor - 1) * kLane];
    if (A.score) A.score[g] = ret;
    for (int f = 0; f < kLatent; ++f)
    {
        const int16_t v = pl[(size_t)f * kLane];
        if (A.latOut) A.latOut[(pl - A.prevLat) + (size_t)f * kLane] = v;   // same [lane][frame][64] layout
        pl[(size_t)f * kLane] = chunk[(size_t)(anchor + f) * kLane];
    }
}

// The lane's old model is replaced by the new one after all its ZMWs used it.
__global__ void LabelerModelCopyKernel(hw_lane_model* dst, const hw_lane_model* src, int lanes, LaneMap map)
{
    constexpr int kWords = (int)(sizeof(hw_lane_model) / 4);
    const int n = map.Lanes(lanes) * kWords;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const size_t w = (size_t)map.Lane(i / kWords) * kWords + i % kWords;
    reinterpret_cast<uint32_t*>(dst)[w] = reinterpret_cast<const uint32_t*>(src)[w];
}

template <bool Mapped, bool Fuse, int Threads, bool Margin = false, bool Grouped = false>
cudaError_t LaunchLabelerT(const LabelerArgs& a, const KParams& k, const PulseArgs& p, int lanes, cudaStream_t s)
{
    const int blocks = (lanes * kLane + Threads - 1) / Threads;
    // ROI words during the forward pass, packed labels after it (fused)
    const int roiWords = (a.F + kLookback + kStitch + 15) / 16;
    const int words = Fuse ? (roiWords > a.F / kBatch ? roiWords : a.F / kBatch) : roiWords;
    const size_t smem = (size_t)words * Threads * sizeof(uint32_t);
    static bool attrSet[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (smem > 48 * 1024 && (dev < 0 || dev >= 64 || !attrSet[dev]))
    {
        e = cudaFuncSetAttribute(LabelerKernel<Mapped, Fuse, Threads, Margin, Grouped>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(((1024 + kLookback + kStitch + 15) / 16 > 1024 / kBatch
                                            ? (1024 + kLookback + kStitch + 15) / 16 : 1024 / kBatch) *
                                       Threads * sizeof(uint32_t)));
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) attrSet[dev] = true;
    }
    LabelerKernel<Mapped, Fuse, Threads, Margin, Grouped><<<blocks, Threads, smem, s>>>(a, k, p);
    return cudaGetLastError();
}

// The generic or the grouped 9-way rows (KParams::grouped9) of one variant.
template <bool Mapped, bool Fuse, int Threads>
cudaError_t LaunchLabelerG(const LabelerArgs& a, const KParams& k, const PulseArgs& p, int lanes, cudaStream_t s)
{
    return k.grouped9 ? LaunchLabelerT<Mapped, Fuse, Threads, false, true>(a, k, p, lanes, s)
                      : LaunchLabelerT<Mapped, Fuse, Threads, false, false>(a, k, p, lanes, s);
}

cudaError_t LaunchLabeler(const LabelerArgs& a, const KParams& k, cudaStream_t s, const PulseArgs* fusedPulses,
                          int lanesPerCta)
{
    if (a.F > 1024 || a.F % kBatch != 0) return cudaErrorInvalidValue;
    const int lanes = a.map.Lanes(a.lanes);
    if (lanes == 0) return cudaSuccess;
    cudaError_t e;
    const PulseArgs none{};
    if (!a.map.On())
    {
        if (fusedPulses || lanesPerCta != 2) return cudaErrorInvalidValue;
        if (a.margin && !a.gap) return cudaErrorInvalidValue;
        e = a.margin ? LaunchLabelerT<false, false, 128, true>(a, k, none, lanes, s)
                     : LaunchLabelerG<false, false, 128>(a, k, none, lanes, s);
    }
    else if (a.margin)
    {
        return cudaErrorInvalidValue;     // margins come from the single-pool labeler
    }
    else if (fusedPulses)
    {
        if (lanesPerCta == 1) e = LaunchLabelerG<true, true, 64>(a, k, *fusedPulses, lanes, s);
        else if (lanesPerCta == 2) e = LaunchLabelerG<true, true, 128>(a, k, *fusedPulses, lanes, s);
        else if (lanesPerCta == 4) e = LaunchLabelerG<true, true, 256>(a, k, *fusedPulses, lanes, s);
        else return cudaErrorInvalidValue;
    }
    else
    {
        if (lanesPerCta == 1) e = LaunchLabelerG<true, false, 64>(a, k, none, lanes, s);
        else if (lanesPerCta == 2) e = LaunchLabelerG<true, false, 128>(a, k, none, lanes, s);
        else if (lanesPerCta == 4) e = LaunchLabelerG<true, false, 256>(a, k, none, lanes, s);
        else return cudaErrorInvalidValue;
    }
    if (e != cudaSuccess) return e;
    const int n = lanes * (int)(sizeof(hw_lane_model) / 4);
    LabelerModelCopyKernel<<<(n + 255) / 256, 256, 0, s>>>(a.latModel, a.models, a.lanes, a.map);
    return cudaGetLastError();
}

}   // namespace hwk
