// Detection-model estimation (grouped-data EM) for sm_100a.
//
// Restates TA/DmeEmHost.cpp:131-852 and TA/DetectionModelHost.cpp:52-285
// (TA = src/basecaller/basecaller/traceAnalysis), with DT/UHistogramSimd.cpp
// Fractile/CumulativeCount.
//
// One CTA of 64 threads per lane, one thread per ZMW.  The reference iterates
// the EM for a whole lane until every ZMW has converged (or failed), and keeps
// blending later iterations into ZMWs that already converged; the lane-wide
// test is a __syncthreads_and, so every ZMW sees exactly the reference's
// iteration sequence.  The E-step keeps the current and previous bin boundary
// in registers; the three per-bin quantities the background-variance M-step
// needs (boundary density, baseline responsibility, n_j / binProb) go to a
// per-lane scratch array in global memory, written and read back coalesced.
#include "hw_device.cuh"

namespace hwk {

__device__ __forceinline__ float pow_d(float x, float y) { return (float)pow((double)x, (double)y); }
__device__ __forceinline__ float exp2_d(float x) { return (float)exp2((double)x); }
__device__ __forceinline__ float log2_d(float x) { return (float)log2((double)x); }

struct ModelF
{
    float bw, bm, bv;
    float aw[kAnalogs], am[kAnalogs], av[kAnalogs];
    float conf;
};

__device__ __forceinline__ void LoadModel(const hw_lane_model& l, int z, ModelF& m)
{
    m.bw = h2f(l.baseline.weights[z]);
    m.bm = h2f(l.baseline.means[z]);
    m.bv = h2f(l.baseline.vars[z]);
#pragma unroll
    for (int a = 0; a < kAnalogs; ++a)
    {
        m.aw[a] = h2f(l.analogs[a].weights[z]);
        m.am[a] = h2f(l.analogs[a].means[z]);
        m.av[a] = h2f(l.analogs[a].vars[z]);
    }
    m.conf = h2f(l.confidence[z]);
}

// ExportTo (DetectionModelHost.cpp:226-234, 277-285)
__device__ __forceinline__ void StoreModel(const ModelF& m, int z, hw_lane_model& l)
{
    const float varMax = h2f(f2h(65000.0f));
    l.baseline.weights[z] = f2h(m.bw);
    l.baseline.means[z] = f2h(m.bm);
    l.baseline.vars[z] = f2h(fmin_sse(m.bv, varMax));
#pragma unroll
    for (int a = 0; a < kAnalogs; ++a)
    {
        l.analogs[a].weights[z] = f2h(m.aw[a]);
        l.analogs[a].means[z] = f2h(m.am[a]);
        l.analogs[a].vars[z] = f2h(fmin_sse(m.av[a], varMax));
    }
    l.confidence[z] = f2h(m.conf);
}

__device__ __forceinline__ float XsnCoeffCVSq(const KParams& k, float mean, float covar, float blVar)
{
    float r = covar - blVar;
    r -= mul_rn(mean, k.shotVarCoeff);
    r /= mul_rn(mean, mean);
    return r;
}

// EvolveConfidence (DetectionModelHost.h:189-201): the confidence decays by
// half every `halfLife` frames between the interval centres.
__device__ __forceinline__ float EvolveConfidence(float conf, int tFrom, int tTo, float halfLife)
{
    const float tDiff = static_cast<float>(tTo - tFrom);
    return mul_rn(conf, exp2_d(-fabsf(tDiff) / halfLife));
}

// DetectionModelHost::Update(other, fraction), Update0/1/2
__device__ void ModelUpdateFrac(const KParams& k, ModelF& t, const ModelF& o, float fraction)
{
    const float a = 1.0f - fraction;
    const float b = fraction;
    if (k.updateMethod == 0)
    {
        t.bm = add_rn(mul_rn(a, t.bm), mul_rn(b, o.bm));
        t.bv = add_rn(mul_rn(a, t.bv), mul_rn(b, o.bv));
        for (int i = 0; i < kAnalogs; ++i)
        {
            t.am[i] = add_rn(mul_rn(a, t.am[i]), mul_rn(b, o.am[i]));
            t.av[i] = add_rn(mul_rn(a, t.av[i]), mul_rn(b, o.av[i]));
        }
        return;
    }
    const float prevBlCovar = t.bv;
    const float bw = add_rn(mul_rn(a, t.bw), mul_rn(b, o.bw));
    t.bw = bw;
    t.bm = add_rn(mul_rn(a, t.bm), mul_rn(b, o.bm));
    const float bv = mul_rn(pow_d(t.bv, a), pow_d(o.bv, b));
    t.bv = bv;
    const float aw = mul_rn(0.25f, 1.0f - bw);
    for (int i = 0; i < kAnalogs; ++i)
    {
        t.aw[i] = aw;
        float cv2;
        if (k.updateMethod == 1) cv2 = k.cv2[i];
        else
        {
            const float tX = XsnCoeffCVSq(k, t.am[i], t.av[i], prevBlCovar);
            const float oX = XsnCoeffCVSq(k, o.am[i], o.av[i], o.bv);
            cv2 = add_rn(mul_rn(a, tX), mul_rn(b, oX));
        }
        const float am = mul_rn(pow_d(t.am[i], a), pow_d(o.am[i], b));
        t.am[i] = am;
        t.av[i] = SignalCovar(k, cv2, am, bv);
    }
}

// DetectionModelHost::Update(other), DetectionModelHost.cpp:207-223
__device__ void ModelUpdate(const KParams& k, ModelF& t, const ModelF& o)
{
    const float confSum = t.conf + o.conf;
    const float frac = (confSum > 0.0f) ? o.conf / confSum : 0.0f;
    ModelUpdateFrac(k, t, o, frac);
    t.conf = confSum;
}

__device__ __forceinline__ float StatMeanD(const hw_stat_accum_state& s, int z)
{
    return s.moment1[z] / s.moment0[z] + s.offset[z];
}

__device__ __forceinline__ float StatVarianceD(const hw_stat_accum_state& s, int z)
{
    const float m0 = s.moment0[z], m1 = s.moment1[z], m2 = s.moment2[z];
    float var = mul_rn(m1, m1) / m0;
    var = (m2 - var) / (m0 - 1.0f);
    var = fmax_sse(var, 0.0f);
    return (m0 > 1.0f) ? var : __int_as_float(0x7fffffff);
}


// Histogram geometry and totals of one ZMW (UHistogramSimd arithmetic in
// uint16 where the reference keeps counts in uint16).
struct EmHist
{
    const hw_lane_histogram* H;
    int z;
    float lb, binSize, varQuant, binProbMin, nSum;
    uint16_t inRange, nLowOut, total;
    // occupied bins of the warp's ZMWs: every bin outside [wLo, wHi] is empty
    // for all of them (wLo > wHi: no occupied bin)
    int wLo, wHi;
    __device__ __forceinline__ float BinStart(int b) const { return add_rn(lb, mul_rn((float)b, binSize)); }
    __device__ __forceinline__ uint32_t Count(int b) const { return H->bin_count[b][z]; }
};

__device__ __forceinline__ void LoadEmHist(const hw_lane_histogram& H, int z, EmHist& h)
{
    h.H = &H;
    h.z = z;
    uint16_t inRange = 0;
    float nSum = 0.0f;
    int lo = kBins, hi = -1;
    for (int b = 0; b < kBins; ++b)
    {
        const uint16_t c = H.bin_count[b][z];
        inRange = (uint16_t)(inRange + c);
        nSum += (float)c;
        lo = (c != 0 && b < lo) ? b : lo;
        hi = (c != 0) ? b : hi;
    }
    h.wLo = __reduce_min_sync(0xffffffffu, lo);
    h.wHi = __reduce_max_sync(0xffffffffu, hi);
    h.inRange = inRange;
    h.nSum = nSum;
    h.nLowOut = H.outlier_count_low[z];
    h.total = (uint16_t)(inRange + (uint16_t)(h.nLowOut + H.outlier_count_high[z]));
    h.lb = H.low_bound[z];
    h.binSize = H.bin_size[z];
    h.varQuant = mul_rn(h.binSize, h.binSize) / 12.0f;
    h.binProbMin = mul_rn(fmax_sse(mul_rn((float)h.total, h.binSize), 1.0f), 1.17549435e-38f);
}

// The EM's free parameters (DmeEmHost.cpp:253-361): mixture fractions, means
// and variances of the baseline and the four analog modes, and the analog
// amplitude scale s (analog means are s * relAmp).
struct EmVars
{
    float rho[5], mu[5], var[5];
    float s;
};

// Regularisation of s toward the preliminary estimate.
struct EmReg
{
    float sExpect, sExpectW;
};

// s of the EM set-up: the relative-amplitude projection of the analog means.
__device__ __forceinline__ float EmScale(const KParams& k, const float mu[5])
{
    const float p0 = mul_rn(mu[1], k.relAmp[0]), p1 = mul_rn(mu[2], k.relAmp[1]);
    const float p2 = mul_rn(mu[3], k.relAmp[2]), p3 = mul_rn(mu[4], k.relAmp[3]);
    return ((p0 + p1) + (p2 + p3)) / k.rpaSum2;
}

// Everything the reference does before its EM iterations: EvolveModel,
// PrelimEstimate and its confidence-weighted update, PrelimScaleFactor,
// ScaleModelSnr and the EM set-up (DmeEmHost.cpp:161-361, 620-654, 806-852).
// Leaves the updated prior model in `det` and the EM start in `v`.
__device__ __forceinline__ void DmePrelude(const KParams& k, const hw_lane_model& M, const hw_baseliner_stats& BS,
                                           const EmHist& h, int tModel, int tEst, ModelF& det, EmVars& v, EmReg& r)
{
    const int z = h.z;
    const hw_lane_histogram& H = *h.H;
    LoadModel(M, z, det);

    // EvolveModel (DmeEmHost.cpp:806-834) + EvolveConfidence (DetectionModelHost.h:166-177)
    {
        const float thl = mul_rn(0.5f, (float)(tModel + tEst));
        const float t0 = 56160.0f, t1 = 168480.0f;
        const float hl = add_rn(k.halfLife0, mul_rn(k.halfLife1 - k.halfLife0, satlin_std(t0, t1, thl)));
        det.conf = EvolveConfidence(det.conf, tModel, tEst, hl);
    }

    // PrelimEstimate (DmeEmHost.cpp:161-214)
    ModelF work = det;
    {
        const float nBl = BS.baseline_stats.moment0[z];
        const float tot = BS.full_autocorr.basic_stats.moment0[z];
        const float blWeight = fmax_sse(nBl / tot, 0.01f);
        const bool mask = nBl >= 3.0f;
        float blVar = mask ? StatVarianceD(BS.baseline_stats, z) : work.bv;
        blVar = fmin_sse(fmax_sse(blVar, k.blVarMin), k.blVarMax);
        const float blMean = mask ? StatMeanD(BS.baseline_stats, z) : work.bm;
        const float scale = sqrtf(blVar / work.bv);
        for (int i = 0; i < kAnalogs; ++i)
        {
            const float mean = mul_rn(work.am[i], scale);
            work.am[i] = mean;
            work.av[i] = SignalCovar(k, k.cv2[i], mean, blVar);
            work.aw[i] = mul_rn(0.25f, 1.0f - blWeight);
        }
        work.bw = blWeight;
        work.bm = blMean;
        work.bv = blVar;
        float conf = mul_rn(0.1f, satlin_sse(0.0f, 500.0f, nBl - 3.0f));
        conf = mul_rn(conf, satlin_sse(k.blVarMax, mul_rn(0.5f, k.blVarNominal + k.blVarMax), blVar));
        work.conf = conf;
    }
    ModelUpdate(k, det, work);
    work = det;

    const float lb = h.lb, binSize = h.binSize;
    const uint16_t nLowOut = h.nLowOut, inRange = h.inRange, total = h.total;

    // PrelimScaleFactor (DmeEmHost.cpp:620-654)
    float scaleFactor;
    {
        const float bgSigma = sqrtf(work.bv);
        const float thresh = add_rn(mul_rn(2.5f, bgSigma), work.bm);
        // CumulativeCount (UHistogramSimd.cpp:204-242)
        float bgCount;
        {
            const float x = thresh;
            const float ub = h.BinStart(kBins);
            const bool mNan = isnan(x), mLow = x < lb, mHigh = x >= ub;
            const bool inB = !(mNan | mLow | mHigh);
            int xbin = floor_cast_i32((x - lb) / binSize);
            xbin = inB ? xbin : 0;
            const float xrem = x - h.BinStart(xbin);
            const float xbinCount = (float)(xbin < kBins ? H.bin_count[xbin][z] : (uint16_t)0);
            float cc = (float)nLowOut;
            uint16_t cn = 0;
            const int lim = xbin < kBins ? xbin : kBins;
            for (int i = 0; i < lim; ++i) cn = (uint16_t)(cn + H.bin_count[i][z]);
            cc += (float)cn;
            cc += mul_rn(xbinCount, xrem) / binSize;
            cc = mLow ? (float)nLowOut : cc;
            cc = mHigh ? (float)(uint16_t)(nLowOut + inRange) : cc;
            cc = mNan ? __int_as_float(0x7fffffff) : cc;
            bgCount = cc;
        }
        const float totalCount = (float)(uint16_t)(nLowOut + inRange);
        const float fractile = mul_rn(0.5f, bgCount + totalCount) / totalCount;
        float avg = 0.0f;
        for (int a = 0; a < kAnalogs; ++a) avg += work.am[a];
        avg /= static_cast<float>(kAnalogs);
        const float w = satlin_sse(0.0f, k.scaleSnrConfTol, work.conf);
        // Fractile (UHistogramSimd.cpp:142-201)
        float frv;
        {
            const float nfz = mul_rn(fractile, (float)total);
            uint16_t n = nLowOut;
            if (n > 0 && n >= nfz) frv = -__int_as_float(0x7f800000);
            else
            {
                int i = 0;
                while ((n == 0 || n < nfz) && i < kBins) n = (uint16_t)(n + H.bin_count[i++][z]);
                if (n < nfz) frv = __int_as_float(0x7f800000);
                else
                {
                    i -= 1;
                    const float x0 = h.BinStart(i);
                    const uint16_t niz = H.bin_count[i][z];
                    const int m = (int)n - (int)niz;
                    frv = add_rn(x0, mul_rn(binSize, nfz - (float)m) / (float)(niz + 1));
                }
            }
        }
        float sf = frv / avg;
        sf = add_rn(mul_rn(1.0f - w, sf), w);
        scaleFactor = fmin_sse(fmax_sse(sf, 0.1f), 10.0f);
    }
    // ScaleModelSnr (DmeEmHost.cpp:837-852)
    for (int a = 0; a < kAnalogs; ++a)
    {
        work.am[a] = mul_rn(scaleFactor, work.am[a]);
        work.av[a] = SignalCovar(k, k.cv2[a], work.am[a], work.bv);
    }

    // EM setup (DmeEmHost.cpp:253-361)
    const float rhoMin = 0.001f;
    v.rho[0] = fmax_sse(work.bw, rhoMin); v.mu[0] = work.bm; v.var[0] = work.bv;
    for (int a = 0; a < kAnalogs; ++a)
    {
        v.rho[a + 1] = fmax_sse(work.aw[a], rhoMin);
        v.mu[a + 1] = work.am[a];
        v.var[a + 1] = work.av[a];
    }
    for (int i = 0; i < 5; ++i) v.var[i] += h.varQuant;
    v.var[0] = fmin_sse(v.var[0], k.blVarMax);
    {
        const float rs = (v.rho[0] + v.rho[1]) + (v.rho[2] + (v.rho[3] + v.rho[4]));
        for (int i = 0; i < 5; ++i) v.rho[i] = v.rho[i] / rs;
    }
    v.s = EmScale(k, v.mu);
    r.sExpect = v.s / scaleFactor;
    r.sExpectW = mul_rn(det.conf, k.pulseAmpReg);
}

// One E-step over the 301 bin boundaries and 300 bins (DmeEmHost.cpp:363-492):
// returns the log-likelihood, fills the mode totals ci, first moments mom1 and
// inverse variances, and writes what the background-variance M-step needs to
// the lane's scratch.
//
// Only bins with a count contribute to c_i, mom1, wps and (in the M-step)
// mom2: an empty bin adds (finite) x 0 = +-0 to sums that start at +0 and
// therefore never hold -0, which leaves them unchanged.  So the
// responsibilities (5 exps), log(binProb) and n_j / binProb are only
// evaluated next to occupied bins; the boundary density, which every bin
// probability needs, is always evaluated.  The shortcut needs every boundary
// density finite: llb <= max(pref) + log(5), so finite prefactors, means and
// inverse variances with max(pref) < 80 guarantee it (`safe`).  Otherwise the
// reference path runs.
//
// kFull = false computes the log-likelihood alone (the same bits): no
// responsibilities, sums or scratch, for the start that is only compared.
template <bool kFull = true>
__device__ __forceinline__ float EmEStep(const KParams& k, const EmHist& h, const EmVars& v, const EmReg& r,
                                         float* bpS, float* tau0S, float* facS, float ci[5], float mom1[5],
                                         float varinv[5], bool& safeOut)
{
    // Modes 0/1 and 2/3 run as packed pairs (hw_expf2, f32x2 arithmetic:
    // each component rounds exactly as the scalar operation), mode 4 alone.
    // Subtractions are additions of the exactly negated operand, and
    // pref - ((0.5 y) y) vinv is pref + ((-0.5 y) y) vinv: the same bits.
    const int z = h.z;
    const float halfLog2pi = mul_rn(0.5f, k.logTwoPi);
    float pref[5];
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        varinv[i] = 1.0f / v.var[i];
        pref[i] = (hw_logf(v.rho[i]) - mul_rn(0.5f, hw_logf(v.var[i]))) - halfLog2pi;
    }
    bool safe = true;
    {
        float pmax = pref[0];
#pragma unroll
        for (int i = 0; i < 5; ++i)
        {
            safe &= isfinite(pref[i]) & isfinite(v.mu[i]) & isfinite(varinv[i]);
            pmax = fmaxf(pmax, pref[i]);
        }
        safe &= pmax < 80.0f;
    }
    const float2 pref01 = f2(pref[0], pref[1]), pref23 = f2(pref[2], pref[3]);
    const float2 vinv01 = f2(varinv[0], varinv[1]), vinv23 = f2(varinv[2], varinv[3]);
    const float2 nmu01 = f2(-v.mu[0], -v.mu[1]), nmu23 = f2(-v.mu[2], -v.mu[3]);
    const float pref4 = pref[4], vinv4 = varinv[4], mu4 = v.mu[4];
    const float2 nz = f2(k.negZero);
    float probSum = 0.0f, wps = 0.0f;
    float2 ci01 = f2(0.0f), ci23 = f2(0.0f), m01 = f2(0.0f), m23 = f2(0.0f);
    float ci4 = 0.0f, m4 = 0.0f;
    float2 tp01 = f2(0.0f), tp23 = f2(0.0f);
    float tp4 = 0.0f, bpPrev = 0.0f, xPrev = 0.0f;
    uint32_t nPrev = 0;
    // bin counts are loaded one boundary ahead of their use
    uint32_t nNext = h.Count(0);
    for (int b = 0; b <= kBins; ++b)
    {
        // cornerComp(b)
        const float x = h.BinStart(b);
        const float2 x2 = f2(x);
        float2 y = add2(x2, nmu01);
        const float2 t01 = add2(pref01, mulz2(mul2(mul2(f2(-0.5f), y), y), vinv01, nz));
        y = add2(x2, nmu23);
        const float2 t23 = add2(pref23, mulz2(mul2(mul2(f2(-0.5f), y), y), vinv23, nz));
        float t4;
        {
            const float y4 = x - mu4;
            t4 = pref4 - mul_rn(mul_rn(mul_rn(0.5f, y4), y4), vinv4);
        }
        float tmax = t01.x;
        tmax = fmax_sse(tmax, t01.y);
        tmax = fmax_sse(tmax, t23.x);
        tmax = fmax_sse(tmax, t23.y);
        tmax = fmax_sse(tmax, t4);
        const uint32_t nCur = nNext;
        nNext = (b + 1 < kBins) ? h.Count(b + 1) : 0u;
        const bool needTau = kFull & ((nPrev != 0u) | (nCur != 0u) | !safe);
        // Far tails: with every t finite and below -106, llb = tmax +
        // log(se) with 1 <= se <= 5 stays below -104.3, where hw_expf
        // returns exactly 0, so bp is 0 without evaluating it.
        // (a finite sum means every t is finite; an infinite or NaN t, or a
        // sum that merely overflows, only forgoes the shortcut)
        const float2 tsum = add2(t01, t23);
        const bool allFinite = isfinite(add_rn(add_rn(tsum.x, tsum.y), t4));
        const bool tail = !needTau & allFinite & (tmax < -106.0f);
        float bp = 0.0f, llb = 0.0f;
        if (!tail)
        {
            const float2 ntmax = f2(-tmax);
            const float2 e01 = hw_expf2_np(add2(t01, ntmax), nz), e23 = hw_expf2_np(add2(t23, ntmax), nz);
            float se = add_rn(e01.x, e01.y);
            se = add_rn(se, e23.x);
            se = add_rn(se, e23.y);
            se = add_rn(se, hw_expf_np(t4 - tmax));
            llb = add_rn(tmax, hw_logf(se));
            bp = hw_expf(llb);
        }
        float2 tau01 = f2(0.0f), tau23 = f2(0.0f);
        float tau4 = 0.0f;
        if (needTau)
        {
            const float2 nllb = f2(-llb);
            tau01 = hw_expf2_np(add2(t01, nllb), nz);
            tau23 = hw_expf2_np(add2(t23, nllb), nz);
            tau4 = hw_expf_np(t4 - llb);
            bpS[(size_t)b * kLane + z] = bp;
            tau0S[(size_t)b * kLane + z] = tau01.x;
        }
        if (b > 0)
        {
            // centerComp(b - 1)
            const int c = b - 1;
            const float bpr = fmax_sse(mul_rn(mul_rn(0.5f, h.binSize), add_rn(bpPrev, bp)), h.binProbMin);
            probSum = add_rn(probSum, bpr);
            if (!kFull && ((nPrev != 0u) | !safe))
                wps = add_rn(wps, mul_rn((float)nPrev, hw_logf(bpr)));
            if (kFull && ((nPrev != 0u) | !safe))
            {
                const float njb = (float)nPrev;
                wps = add_rn(wps, mul_rn(njb, hw_logf(bpr)));
                const float factor = njb / bpr;
                facS[(size_t)c * kLane + z] = factor;
                const float2 fac = f2(factor), bpp = f2(bpPrev), bpc = f2(bp), xp = f2(xPrev);
                float2 tmp1 = mulz2(bpp, tp01, nz), tmp2 = mulz2(bpc, tau01, nz);
                ci01 = add2(ci01, mulz2(add2(tmp1, tmp2), fac, nz));
                m01 = add2(m01, mulz2(add2(mulz2(tmp1, xp, nz), mulz2(tmp2, x2, nz)), fac, nz));
                tmp1 = mulz2(bpp, tp23, nz);
                tmp2 = mulz2(bpc, tau23, nz);
                ci23 = add2(ci23, mulz2(add2(tmp1, tmp2), fac, nz));
                m23 = add2(m23, mulz2(add2(mulz2(tmp1, xp, nz), mulz2(tmp2, x2, nz)), fac, nz));
                const float s1 = mul_rn(bpPrev, tp4), s2 = mul_rn(bp, tau4);
                ci4 = add_rn(ci4, mul_rn(add_rn(s1, s2), factor));
                m4 = add_rn(m4, mul_rn(add_rn(mul_rn(s1, xPrev), mul_rn(s2, x)), factor));
            }
        }
        tp01 = tau01;
        tp23 = tau23;
        tp4 = tau4;
        bpPrev = bp;
        xPrev = x;
        nPrev = nCur;
    }
    const float2 hb = f2(mul_rn(0.5f, h.binSize));
    ci01 = mulz2(ci01, hb, nz);
    ci23 = mulz2(ci23, hb, nz);
    m01 = mulz2(m01, hb, nz);
    m23 = mulz2(m23, hb, nz);
    ci[0] = ci01.x; ci[1] = ci01.y; ci[2] = ci23.x; ci[3] = ci23.y; ci[4] = mul_rn(ci4, hb.x);
    mom1[0] = m01.x; mom1[1] = m01.y; mom1[2] = m23.x; mom1[3] = m23.y; mom1[4] = mul_rn(m4, hb.x);
    float ll = wps - mul_rn(h.nSum, hw_logf(probSum));
    const float ds = v.s - r.sExpect;
    ll = ll - mul_rn(mul_rn(0.5f, mul_rn(ds, ds)), r.sExpectW);
    safeOut = safe;
    return ll;
}

// One M-step (DmeEmHost.cpp:494-565) from the E-step's sums; ci is floored in
// place.  Sets bit 4 (VLOW_SIGNAL) of zStatus when s is clamped to its floor.
__device__ __forceinline__ void EmMStep(const KParams& k, const EmHist& h, const EmReg& r, bool safe,
                                        const float* bpS, const float* tau0S, const float* facS, float ci[5],
                                        const float mom1[5], const float varinv[5], EmVars& v, int& zStatus)
{
    const int z = h.z;
#pragma unroll
    for (int i = 0; i < 5; ++i) ci[i] = fmax_sse(ci[i], 0.1f);
#pragma unroll
    for (int i = 0; i < 5; ++i) v.rho[i] = ci[i] / h.nSum;
    {
        const float rs = (v.rho[0] + v.rho[1]) + (v.rho[2] + (v.rho[3] + v.rho[4]));
#pragma unroll
        for (int i = 0; i < 5; ++i) v.rho[i] = v.rho[i] / rs;
    }
    v.mu[0] = mom1[0] / ci[0];
    float numer = 0.0f, denom = 0.0f;
#pragma unroll
    for (int a = 0; a < kAnalogs; ++a)
    {
        const int i = a + 1;
        numer = add_rn(numer, mul_rn(mul_rn(k.relAmp[a], varinv[i]), mom1[i]));
        denom = add_rn(denom, mul_rn(mul_rn(mul_rn(k.relAmp[a], k.relAmp[a]), varinv[i]), ci[i]));
    }
    numer = add_rn(numer, mul_rn(r.sExpect, r.sExpectW));
    denom = add_rn(denom, r.sExpectW);
    float sv = numer / denom;
    const float sMin = fmax_sse(mul_rn(0.5f, sqrtf(v.var[0])), k.minPulseMean) / k.rpaMin;
    const bool vls = sv < sMin;
    sv = vls ? sMin : sv;
    if (vls) zStatus |= 4;
    v.s = sv;
#pragma unroll
    for (int a = 0; a < kAnalogs; ++a) v.mu[a + 1] = mul_rn(sv, k.relAmp[a]);
    // Background variance: second pass over the bins.  The scratch values of
    // boundary j + 1 are those of boundary j in the next bin, so each is
    // loaded once, one bin ahead of its use.  Scratch slots of boundaries next
    // to empty bins hold stale values; they are loaded but only used for
    // occupied bins (or when !safe, where every boundary was written).
    // Bins that are empty for every ZMW of the warp add +0 to every sum (see
    // the E-step), so when all of the warp's ZMWs are `safe` the pass covers
    // only the warp's occupied range.
    float mom2 = 0.0f;
    {
        const bool narrow = __all_sync(0xffffffffu, safe);
        const int j0 = narrow ? h.wLo : 0;
        const int j1 = narrow ? h.wHi + 1 : kBins;
        float bpj = 0.0f, t0j = 0.0f;
        uint32_t nj = 0u;
        if (j0 < j1)
        {
            bpj = bpS[(size_t)j0 * kLane + z];
            t0j = tau0S[(size_t)j0 * kLane + z];
            nj = h.Count(j0);
        }
        for (int j = j0; j < j1; ++j)
        {
            const float bpk = bpS[(size_t)(j + 1) * kLane + z], t0k = tau0S[(size_t)(j + 1) * kLane + z];
            const float fj = facS[(size_t)j * kLane + z];
            const uint32_t nk = (j + 1 < kBins) ? h.Count(j + 1) : 0u;
            if (!safe || nj != 0u)      // an empty bin adds +0 (see the E-step)
            {
                const float xj = h.BinStart(j) - v.mu[0];
                const float xk = h.BinStart(j + 1) - v.mu[0];
                float tmp = mul_rn(mul_rn(mul_rn(bpj, xj), xj), t0j);
                tmp = add_rn(tmp, mul_rn(mul_rn(mul_rn(bpk, xk), xk), t0k));
                tmp = mul_rn(tmp, fj);
                mom2 = add_rn(mom2, tmp);
            }
            bpj = bpk;
            t0j = t0k;
            nj = nk;
        }
    }
    mom2 = mul_rn(mom2, mul_rn(0.5f, h.binSize));
    float v0 = add_rn(mom2 / ci[0], h.varQuant);
    v0 = fmin_sse(fmax_sse(v0, k.blVarMin), k.blVarMax);
    v.var[0] = v0;
#pragma unroll
    for (int a = 0; a < kAnalogs; ++a) v.var[a + 1] = SignalCovar(k, k.cv2[a], v.mu[a + 1], v0);
}

// The learned start: replaces the reference start v by the proposal column Q
// unless the proposal's log-likelihood is lower (or not comparable); returns
// 1 when it kept the reference start.  Reports both log-likelihoods.  The
// proposal's E-step is the full one and the reference start's only its
// log-likelihood, so when the proposal is kept, ci/mom1/varinv/safe and the
// per-bin scratch hold its E-step, which is the first EM iteration's E-step
// from that start.
__device__ __forceinline__ int ChooseStart(const KParams& k, const EmHist& h, const EmReg& r, const float* Q, bool fallback,
                                           float* bpS, float* tau0S, float* facS, EmVars& v, float& llPlain,
                                           float& llStart, float (&ci)[5], float (&mom1)[5], float (&varinv)[5],
                                           bool& safe)
{
    const int z = h.z;
    EmVars p;
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        p.rho[i] = Q[i * kLane + z];
        p.mu[i] = Q[(5 + i) * kLane + z];
        p.var[i] = Q[(10 + i) * kLane + z];
    }
    p.s = EmScale(k, p.mu);
    const float llProp = EmEStep(k, h, p, r, bpS, tau0S, facS, ci, mom1, varinv, safe);
    {
        float ciX[5], momX[5], vinvX[5];
        bool safeX;
        llPlain = EmEStep<false>(k, h, v, r, bpS, tau0S, facS, ciX, momX, vinvX, safeX);
    }
    llStart = llPlain;
    if (fallback && !(llProp >= llPlain)) return 1;
    v = p;
    llStart = llProp;
    return 0;
}

// Learned: the start comes from A.proposal (with the fallback test); Clock:
// the per-lane phase clock of A.phases.  Both are compile-time so that the
// reference-start variant carries neither the start choice's values nor the
// clock's counters through its EM loop (they cost registers there).
template <bool Mapped, bool Learned, bool Clock>
__global__ void __launch_bounds__(kLane, 10) DmeEstimateKernel(DmeArgs A, KParams k)
{
    LaneMap map = A.map;
    if (!Mapped) map.list = nullptr;      // the single-pool variant compiles without the lane list
    // scratch belongs to the launch lane, the rest to the (engine) lane
    const int li = blockIdx.x;
    const int l = map.Lane(li);
    const int z = threadIdx.x;
    int32_t tModel = A.tModel, tEst = A.tEst;
    if (map.On())
    {
        const PoolStep& ps = map.Pool(l);
        tModel = ps.tModel;
        tEst = ps.tEst;
    }
    float* bpS = A.scratch + (size_t)li * 3 * (kBins + 1) * kLane;
    float* tau0S = bpS + (size_t)(kBins + 1) * kLane;
    float* facS = tau0S + (size_t)(kBins + 1) * kLane;

    // phase clock (thread 0, when asked for): see DmeArgs::phases
    const bool clk = Clock && z == 0;
    long long tc[5] = {0, 0, 0, 0, 0};
    long long tMark = clk ? clock64() : 0;
    const long long tBegin = tMark;
    auto lap = [&](int phase) {
        if (clk)
        {
            const long long t = clock64();
            tc[phase] += t - tMark;
            tMark = t;
        }
    };

    EmHist h;
    LoadEmHist(A.hist[l], z, h);
    ModelF det;
    EmVars v;
    EmReg r;
    DmePrelude(k, A.models[l], A.stats[l], h, tModel, tEst, det, v, r);
    lap(0);
    // Values needed only before and after the EM iterations (the prior model
    // and the estimates at the latest converged iteration) wait in per-thread
    // shared-memory columns, which keeps them out of registers in the loop.
    __shared__ float shDet[16][kLane];
    __shared__ float shEst[15][kLane];
    auto rhoEst = [&](int i) -> float& { return shEst[i][z]; };
    auto muEst = [&](int i) -> float& { return shEst[5 + i][z]; };
    auto varEst = [&](int i) -> float& { return shEst[10 + i][z]; };
    for (int i = 0; i < 5; ++i) { rhoEst(i) = v.rho[i]; muEst(i) = v.mu[i]; varEst(i) = v.var[i]; }

    // The learned start (the same decisions as ChooseStart): the reference
    // start's log-likelihood alone, then the proposal's full E-step, which
    // becomes the first iteration's E-step when the proposal is kept.  The
    // reference start waits in shEst meanwhile (its scale is EmScale of its
    // means, as DmePrelude sets it), so only one start is in registers.
    float ci[5], mom1[5], varinv[5];
    bool safe = false, haveE = false;
    float llE = 0.0f;
    int fellBack = 0;
    if constexpr (Learned)
    {
        float llPlain;
        {
            float ciX[5], momX[5], vinvX[5];
            bool safeX;
            llPlain = EmEStep<false>(k, h, v, r, bpS, tau0S, facS, ciX, momX, vinvX, safeX);
        }
        const float* Q = A.proposal + (size_t)l * 15 * kLane;
#pragma unroll
        for (int i = 0; i < 5; ++i)
        {
            v.rho[i] = Q[i * kLane + z];
            v.mu[i] = Q[(5 + i) * kLane + z];
            v.var[i] = Q[(10 + i) * kLane + z];
        }
        v.s = EmScale(k, v.mu);
        const float llProp = EmEStep(k, h, v, r, bpS, tau0S, facS, ci, mom1, varinv, safe);
        haveE = llProp >= llPlain;
        if (haveE)
        {
            llE = llProp;
            for (int i = 0; i < 5; ++i) { rhoEst(i) = v.rho[i]; muEst(i) = v.mu[i]; varEst(i) = v.var[i]; }
        }
        else
        {
#pragma unroll
            for (int i = 0; i < 5; ++i) { v.rho[i] = rhoEst(i); v.mu[i] = muEst(i); v.var[i] = varEst(i); }
            v.s = EmScale(k, v.mu);
        }
        fellBack = __syncthreads_count(!haveE);
    }
    lap(1);
    {
        shDet[0][z] = det.bw; shDet[1][z] = det.bm; shDet[2][z] = det.bv; shDet[3][z] = det.conf;
#pragma unroll
        for (int a = 0; a < kAnalogs; ++a)
        {
            shDet[4 + a][z] = det.aw[a]; shDet[8 + a][z] = det.am[a]; shDet[12 + a][z] = det.av[a];
        }
    }
    float logLike = -3.40282347e+38f;
    int zStatus = (h.total < 160u) ? 2 : 0;
    bool mConverged = false;
    int mIter = 0;
    float mLogLike = -__int_as_float(0x7f800000);

    const int iterLimit = k.emIterLimit;
    int it = 0;
    // An EM iteration after its E-step (log-likelihood ll): convergence
    // bookkeeping, the lane vote and the M-step; true when the lane stops.
    auto finishIteration = [&](float ll) -> bool {
        const float prev = logLike;
        logLike = ll;
        const float delta = ll - prev;
        const float convTol = mul_rn(1e-4f, fmax_sse(ll, -ll));
        bool cv = (delta >= 0) & (delta < convTol);
        cv &= (ll >= mLogLike);
        mIter = (cv & !mConverged) ? it : mIter;
        mLogLike = cv ? ll : mLogLike;
        mConverged |= cv;
        if (cv)
        {
#pragma unroll
            for (int i = 0; i < 5; ++i) { rhoEst(i) = v.rho[i]; muEst(i) = v.mu[i]; varEst(i) = v.var[i]; }
        }
        const int allDone = __syncthreads_and(mConverged | (zStatus != 0));
        lap(2);
        if (!k.iterToLimit && allDone) return true;
        EmMStep(k, h, r, safe, bpS, tau0S, facS, ci, mom1, varinv, v, zStatus);
        lap(3);
        return false;
    };
    bool stopped = false;
    if constexpr (Learned)
    {
        // the first iteration apart: a kept proposal's E-step is already done
        // (peeled, so its values are not carried around the loop)
        if (it < iterLimit)
        {
            const float ll = haveE ? llE : EmEStep(k, h, v, r, bpS, tau0S, facS, ci, mom1, varinv, safe);
            stopped = finishIteration(ll);
            if (!stopped) ++it;
        }
    }
    if (!stopped)
        for (; it < iterLimit; ++it)
            if (finishIteration(EmEStep(k, h, v, r, bpS, tau0S, facS, ci, mom1, varinv, safe))) break;
    const int laneIters = it + 1 < iterLimit ? it + 1 : iterLimit;

    if (!mConverged) zStatus |= 1;
    bool finite = true;
#pragma unroll
    for (int i = 0; i < 5; ++i) finite &= isfinite(rhoEst(i)) & isfinite(muEst(i)) & isfinite(varEst(i));
    ModelF work;
    work.bw = rhoEst(0); work.bm = muEst(0); work.bv = varEst(0);
#pragma unroll
    for (int a = 0; a < kAnalogs; ++a) { work.aw[a] = rhoEst(a + 1); work.am[a] = muEst(a + 1); work.av[a] = varEst(a + 1); }
    {
        det.bw = shDet[0][z]; det.bm = shDet[1][z]; det.bv = shDet[2][z]; det.conf = shDet[3][z];
#pragma unroll
        for (int a = 0; a < kAnalogs; ++a)
        {
            det.aw[a] = shDet[4 + a][z]; det.am[a] = shDet[8 + a][z]; det.av[a] = shDet[12 + a][z];
        }
    }
    if (!finite) atomicCAS(A.err, 0, HW_ERR_NUMERIC);

    // ComputeConfidence (DmeEmHost.cpp:717-803), G-test disabled (pValue 1)
    float conf;
    {
        float cf[7];
        cf[0] = mConverged ? 1.0f : 0.0f;
        cf[1] = satlin_sse(0.05f, 0.15f, work.bw);
        float x = mul_rn(work.bm, work.bm) / work.bv;
        x = hw_expf(-x / 2.0f);
        cf[2] = x;
        x = log2_d(work.bv / det.bv);
        const float bgVarTol = 1.5f / (0.5f + det.conf);
        x = hw_expf(mul_rn(-x, x) / mul_rn(2.0f, mul_rn(bgVarTol, bgVarTol)));
        cf[3] = x;
        x = 1.0f;
        if (k.amft1 > 0.0f)
        {
            x = mul_rn(x, satlin_sse(k.amft0, k.amft1, work.aw[0]));
            x = mul_rn(x, satlin_sse(k.amft0, k.amft1, work.aw[kAnalogs - 1]));
        }
        cf[4] = x;
        x = work.am[kAnalogs - 1];
        const float bgSigma = sqrtf(work.bv);
        x = x / bgSigma;
        cf[5] = satlin_sse(k.snrThresh0, k.snrThresh1, x);
        if (k.snrDropThresh < 0.0f) cf[6] = 1.0f;
        else
        {
            const float snrEst = work.am[0] / bgSigma;
            const float r0 = det.am[0], r1 = det.am[1];
            const float refBgSigma = sqrtf(det.bv);
            bool ok = (r0 >= 0.0f) & (r1 >= 0.0f) & (refBgSigma >= 0.0f);
            const float refSnr0 = r0 / refBgSigma;
            float refSnr1 = r1 / refBgSigma;
            refSnr1 = mul_rn(refSnr1, k.snrDropThresh);
            refSnr1 = mul_rn(refSnr1, fmin_sse(det.conf, 1.0f));
            ok &= (refSnr1 < refSnr0);
            if (!ok) atomicCAS(A.err, 0, HW_ERR_NUMERIC);
            cf[6] = satlin_sse(refSnr1, sqrtf(mul_rn(refSnr0, refSnr1)), snrEst);
        }
        float cc = 1.0f;
#pragma unroll
        for (int i = 0; i < 7; ++i) cc = mul_rn(cc, cf[i]);
        cc = mul_rn(cc, 1.0f);     // G_TEST factor (pValue == 1)
        cc = fmin_sse(fmax_sse(0.0f, cc), 1.0f);
        cc = (cc >= k.successConfThresh) ? cc : 0.0f;
        conf = cc;
        work.conf = cc;
    }
    ModelUpdate(k, det, work);
    StoreModel(det, z, A.models[l]);
    if (A.diag)
    {
        hw_dme_diag& D = A.diag[l];
        D.iter_count[z] = mIter;
        D.converged[z] = mConverged ? 1 : 0;
        D.log_like[z] = mLogLike;
        D.status[z] = zStatus;
        D.confidence[z] = conf;
        if (z == 0) D.lane_iterations = laneIters;
        if (z < 15) D.pad_[z] = 0;
    }
    if (clk)
    {
        lap(4);
        long long* P = A.phases + (size_t)li * 8;
#pragma unroll
        for (int i = 0; i < 5; ++i) P[i] = tc[i];
        P[5] = laneIters;
        P[6] = tMark - tBegin;
        P[7] = fellBack;
    }
}

cudaError_t LaunchDmeEstimate(const DmeArgs& a, const KParams& k, cudaStream_t s)
{
    const int blocks = a.map.Lanes(a.lanes);
    if (blocks == 0) return cudaSuccess;
    const bool learned = a.proposal != nullptr, clock = a.phases != nullptr;
    if (a.map.On())
    {
        if (learned) DmeEstimateKernel<true, true, false><<<blocks, kLane, 0, s>>>(a, k);
        else DmeEstimateKernel<true, false, false><<<blocks, kLane, 0, s>>>(a, k);
    }
    else if (!clock)
    {
        if (learned) DmeEstimateKernel<false, true, false><<<blocks, kLane, 0, s>>>(a, k);
        else DmeEstimateKernel<false, false, false><<<blocks, kLane, 0, s>>>(a, k);
    }
    else
    {
        if (learned) DmeEstimateKernel<false, true, true><<<blocks, kLane, 0, s>>>(a, k);
        else DmeEstimateKernel<false, false, true><<<blocks, kLane, 0, s>>>(a, k);
    }
    return cudaGetLastError();
}

// ---- Single-ZMW EM fit (learned initializer) ------------------------------------
// The reference's EM steps for each ZMW on its own: from the plain start of
// DmePrelude, from a caller's proposal, or from whichever of the two has the
// higher log-likelihood; maxIter iterations for every ZMW (no lane-wide stop)
// and no final confidence blend.  Records the first iteration that meets the
// reference's convergence test and the first iteration whose parameters lie
// within `tol` of a target.  No counterpart in the reference.
struct DmeFitArgs
{
    const hw_lane_histogram* hist;
    const hw_baseliner_stats* stats;
    const hw_lane_model* models;
    const float* proposal;     // [lanes][15][64] or null
    const float* target;       // [lanes][15][64] or null
    float* scratch;            // [lanes][3][301][64]
    float* params;             // [lanes][15][64]
    int32_t* iters;            // [lanes][5][64]
    float* loglike;            // [lanes][3][64]
    int lanes, tModel, tEst, mode, maxIter;
    float tol;
    float* atStop = nullptr;   // [lanes][15][64] or null: parameters at the first converged iteration
};

// Largest relative distance of the parameters from a target column, with
// floors 0.01 (fractions), 1 DN (means) and 1 DN^2 (variances).
__device__ __forceinline__ float EmDistance(const EmVars& v, const float* t, int z)
{
    float d = 0.0f;
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        const float tr = t[i * kLane + z], tm = t[(5 + i) * kLane + z], tv = t[(10 + i) * kLane + z];
        d = fmaxf(d, fabsf(v.rho[i] - tr) / fmaxf(fabsf(tr), 0.01f));
        d = fmaxf(d, fabsf(v.mu[i] - tm) / fmaxf(fabsf(tm), 1.0f));
        d = fmaxf(d, fabsf(v.var[i] - tv) / fmaxf(fabsf(tv), 1.0f));
    }
    return d;
}

// Largest relative change between two parameter sets (same floors).
__device__ __forceinline__ float EmStep(const EmVars& a, const EmVars& b)
{
    float d = 0.0f;
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        d = fmaxf(d, fabsf(a.rho[i] - b.rho[i]) / fmaxf(fabsf(a.rho[i]), 0.01f));
        d = fmaxf(d, fabsf(a.mu[i] - b.mu[i]) / fmaxf(fabsf(a.mu[i]), 1.0f));
        d = fmaxf(d, fabsf(a.var[i] - b.var[i]) / fmaxf(fabsf(a.var[i]), 1.0f));
    }
    return d;
}

__global__ void __launch_bounds__(kLane, 12) DmeEmFitKernel(DmeFitArgs A, KParams k)
{
    const int l = blockIdx.x;
    const int z = threadIdx.x;
    float* bpS = A.scratch + (size_t)l * 3 * (kBins + 1) * kLane;
    float* tau0S = bpS + (size_t)(kBins + 1) * kLane;
    float* facS = tau0S + (size_t)(kBins + 1) * kLane;

    EmHist h;
    LoadEmHist(A.hist[l], z, h);
    ModelF det;
    EmVars v;
    EmReg r;
    DmePrelude(k, A.models[l], A.stats[l], h, A.tModel, A.tEst, det, v, r);

    float ci[5], mom1[5], varinv[5];
    bool safe;
    float llPlain, llStart;
    int fellBack = 0;
    if (A.mode != HW_EM_START_PLAIN)
        fellBack = ChooseStart(k, h, r, A.proposal + (size_t)l * 15 * kLane, A.mode == HW_EM_START_BETTER, bpS, tau0S,
                               facS, v, llPlain, llStart, ci, mom1, varinv, safe);
    else
    {
        llPlain = EmEStep(k, h, v, r, bpS, tau0S, facS, ci, mom1, varinv, safe);
        llStart = llPlain;
    }
    const float* T = A.target ? A.target + (size_t)l * 15 * kLane : nullptr;
    int zStatus = (h.total < 160u) ? 2 : 0;
    int tolIter = -1, stepIter = -1, mIter = 0;
    bool mConverged = false;
    float logLike = -3.40282347e+38f, mLogLike = -__int_as_float(0x7f800000), last = llStart;
    for (int it = 0; it < A.maxIter; ++it)
    {
        if (T && tolIter < 0 && EmDistance(v, T, z) <= A.tol) tolIter = it;
        const float ll = EmEStep(k, h, v, r, bpS, tau0S, facS, ci, mom1, varinv, safe);
        const float prev = logLike;
        logLike = ll;
        const float delta = ll - prev;
        const float convTol = mul_rn(1e-4f, fmax_sse(ll, -ll));
        bool cv = (delta >= 0) & (delta < convTol);
        cv &= (ll >= mLogLike);
        mIter = (cv & !mConverged) ? it : mIter;
        if (A.atStop && cv && !mConverged)
        {
            // the estimate the reference keeps at its first converged iteration
            float* S = A.atStop + (size_t)l * 15 * kLane;
#pragma unroll
            for (int i = 0; i < 5; ++i)
            {
                S[i * kLane + z] = v.rho[i];
                S[(5 + i) * kLane + z] = v.mu[i];
                S[(10 + i) * kLane + z] = v.var[i];
            }
        }
        mLogLike = cv ? ll : mLogLike;
        mConverged |= cv;
        last = ll;
        const EmVars before = v;
        EmMStep(k, h, r, safe, bpS, tau0S, facS, ci, mom1, varinv, v, zStatus);
        if (stepIter < 0 && EmStep(v, before) <= A.tol) stepIter = it + 1;
    }
    if (T && tolIter < 0 && EmDistance(v, T, z) <= A.tol) tolIter = A.maxIter;
    if (A.atStop && !mConverged)
    {
        float* S = A.atStop + (size_t)l * 15 * kLane;
#pragma unroll
        for (int i = 0; i < 15; ++i) S[i * kLane + z] = __int_as_float(0x7fffffff);
    }

    float* P = A.params + (size_t)l * 15 * kLane;
#pragma unroll
    for (int i = 0; i < 5; ++i)
    {
        P[i * kLane + z] = v.rho[i];
        P[(5 + i) * kLane + z] = v.mu[i];
        P[(10 + i) * kLane + z] = v.var[i];
    }
    int32_t* I = A.iters + (size_t)l * 5 * kLane;
    I[0 * kLane + z] = mConverged ? mIter : -1;
    I[1 * kLane + z] = tolIter;
    I[2 * kLane + z] = fellBack;
    I[3 * kLane + z] = zStatus;
    I[4 * kLane + z] = stepIter;
    float* L = A.loglike + (size_t)l * 3 * kLane;
    L[0 * kLane + z] = llPlain;
    L[1 * kLane + z] = llStart;
    L[2 * kLane + z] = last;
}

// ---- Estimate without device allocation -------------------------------------
// Callers such as a pre-allocated real-time pipeline or code running inside a
// custom allocator's callbacks may not be allowed to call cudaMalloc.  For
// them hw_dme_estimate_noalloc keeps the EM's per-bin scratch in this fixed
// file-scope array instead of a handle-owned allocation.  Every GPU that
// loads the library holds it (about 28 MiB) until the process exits.
constexpr uint32_t kNoAllocMaxLanes = 128;
constexpr size_t kDmeScratchFloatsPerLane = (size_t)3 * (kBins + 1) * kLane;
static __device__ __align__(256) float g_dmeNoAllocScratch[kNoAllocMaxLanes * kDmeScratchFloatsPerLane];
static __device__ __align__(256) int g_dmeNoAllocErr[64];

}   // namespace hwk

#include <mutex>

extern "C" int hw_dme_estimate_noalloc(const hw_config* cfg, uint32_t lanes, const hw_lane_histogram* d_hist,
                                       const hw_baseliner_stats* d_stats, hw_frame_interval hist_fi,
                                       hw_frame_interval model_fi, hw_lane_model* d_models, hw_dme_diag* d_diag,
                                       void* stream)
{
    using namespace hwk;
    if (!cfg || !d_hist || !d_stats || !d_models) return SetLastError(HW_ERR_INVALID_ARG, "NULL argument");
    if (lanes == 0 || lanes > kNoAllocMaxLanes)
        return SetLastError(HW_ERR_INVALID_ARG,
                            "hw_dme_estimate_noalloc: lanes must be in [1, 128]; split larger pools into calls of at most 128 lanes");
    if (hist_fi.lower == hist_fi.upper || model_fi.lower == model_fi.upper)
        return SetLastError(HW_ERR_INVALID_ARG, "frame intervals must not be empty");
    hwp::Derived d;
    KParams k;
    int rc = PrepareConfigNoAlloc(cfg, &d, &k);
    if (rc) return rc;

    // Device addresses of the file-scope arrays, looked up once per device
    // with that device current (host code cannot use the symbols directly).
    static std::mutex mu;
    static float* scratch[64] = {};
    static int* err[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
        return SetLastError(HW_ERR_CUDA, "hw_dme_estimate_noalloc: no current CUDA device");
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!scratch[dev])
        {
            float* p = nullptr;
            int* e = nullptr;
            cudaError_t ce = cudaGetSymbolAddress((void**)&p, g_dmeNoAllocScratch);
            if (ce == cudaSuccess) ce = cudaGetSymbolAddress((void**)&e, g_dmeNoAllocErr);
            if (ce != cudaSuccess)
                return SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
            scratch[dev] = p;
            err[dev] = e;
        }
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // The error word keeps the previous call's value: clear it first.  The
    // scratch needs no clearing: every bin is written before it is read.
    cudaError_t ce = cudaMemsetAsync(err[dev], 0, sizeof(int), s);
    if (ce != cudaSuccess) return SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
    DmeArgs a{d_hist, d_stats, d_models, d_diag, scratch[dev], err[dev], (int)lanes,
              model_fi.lower + (model_fi.upper - model_fi.lower) / 2,
              hist_fi.lower + (hist_fi.upper - hist_fi.lower) / 2};
    ce = LaunchDmeEstimate(a, k, s);
    if (ce != cudaSuccess) return SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
    int h = 0;
    ce = cudaMemcpyAsync(&h, err[dev], sizeof(int), cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    if (ce != cudaSuccess) return SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
    if (h) return SetLastError(h, "DME: a reference sanity assertion failed (non-finite estimate or bad SNR-drop threshold)");
    return HW_OK;
}

extern "C" int hw_dme_em_fit_scratch_bytes(uint32_t lanes, uint64_t* bytes)
{
    if (!bytes) return hwk::SetLastError(HW_ERR_INVALID_ARG, "bytes is NULL");
    *bytes = (uint64_t)lanes * hwk::kDmeScratchFloatsPerLane * sizeof(float);
    return HW_OK;
}

extern "C" int hw_dme_em_fit(const hw_config* cfg, uint32_t lanes, const hw_lane_histogram* d_hist,
                             const hw_baseliner_stats* d_stats, hw_frame_interval hist_fi,
                             hw_frame_interval model_fi, const hw_lane_model* d_models, int start,
                             const float* d_proposal, const float* d_target, float tol, uint32_t max_iter,
                             float* d_scratch, float* d_params, int32_t* d_iters, float* d_loglike,
                             float* d_params_at_stop, void* stream)
{
    using namespace hwk;
    if (!cfg || !d_hist || !d_stats || !d_models || !d_scratch || !d_params || !d_iters || !d_loglike)
        return SetLastError(HW_ERR_INVALID_ARG, "NULL argument");
    if (start < HW_EM_START_PLAIN || start > HW_EM_START_BETTER)
        return SetLastError(HW_ERR_INVALID_ARG, "hw_dme_em_fit: start must be HW_EM_START_PLAIN, _PROPOSAL or _BETTER");
    if (start != HW_EM_START_PLAIN && !d_proposal)
        return SetLastError(HW_ERR_INVALID_ARG, "hw_dme_em_fit: a proposal start needs d_proposal");
    if (lanes == 0 || max_iter > 100000)
        return SetLastError(HW_ERR_INVALID_ARG, "hw_dme_em_fit: lanes must be positive and max_iter at most 100000");
    if (hist_fi.lower == hist_fi.upper || model_fi.lower == model_fi.upper)
        return SetLastError(HW_ERR_INVALID_ARG, "frame intervals must not be empty");
    hwp::Derived d;
    KParams k;
    int rc = PrepareConfigNoAlloc(cfg, &d, &k);
    if (rc) return rc;
    DmeFitArgs a{d_hist, d_stats, d_models, d_proposal, d_target, d_scratch, d_params, d_iters, d_loglike,
                 (int)lanes, model_fi.lower + (model_fi.upper - model_fi.lower) / 2,
                 hist_fi.lower + (hist_fi.upper - hist_fi.lower) / 2, start, (int)max_iter, tol};
    a.atStop = d_params_at_stop;
    DmeEmFitKernel<<<lanes, kLane, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a, k);
    const cudaError_t ce = cudaGetLastError();
    if (ce != cudaSuccess) return SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
    return HW_OK;
}

// ---- DetectionModelHost <-> LaneDetectionModel ------------------------------
// The float model the estimator works on and the fp16 lane model it exports
// (DetectionModelHost(ldm, fi), DetectionModelHost.cpp:47-60; ExportTo,
// DetectionModelHost.cpp:226-234, 277-285), with the DME's own conversion
// functions, so the conversion can be checked on its own.  Float parameters
// are [lane][16][64]: baseline weight, mean, variance; each analog's weight,
// mean, variance; confidence.

namespace hwk {

__global__ void ModelImportKernel(const hw_lane_model* m, float* p, int lanes)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= lanes * kLane) return;
    const int l = g / kLane, z = g % kLane;
    ModelF f;
    LoadModel(m[l], z, f);
    float* o = p + (size_t)l * 16 * kLane + z;
    o[0 * kLane] = f.bw; o[1 * kLane] = f.bm; o[2 * kLane] = f.bv;
    for (int a = 0; a < kAnalogs; ++a)
    {
        o[(3 + 3 * a) * kLane] = f.aw[a];
        o[(4 + 3 * a) * kLane] = f.am[a];
        o[(5 + 3 * a) * kLane] = f.av[a];
    }
    o[15 * kLane] = f.conf;
}

__global__ void ModelExportKernel(const float* p, hw_lane_model* m, int lanes)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= lanes * kLane) return;
    const int l = g / kLane, z = g % kLane;
    const float* i = p + (size_t)l * 16 * kLane + z;
    ModelF f;
    f.bw = i[0 * kLane]; f.bm = i[1 * kLane]; f.bv = i[2 * kLane];
    for (int a = 0; a < kAnalogs; ++a)
    {
        f.aw[a] = i[(3 + 3 * a) * kLane];
        f.am[a] = i[(4 + 3 * a) * kLane];
        f.av[a] = i[(5 + 3 * a) * kLane];
    }
    f.conf = i[15 * kLane];
    StoreModel(f, z, m[l]);
}

__global__ void ModelEvolveKernel(float* p, int lanes, int tFrom, int tTo, float halfLife)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= lanes * kLane) return;
    float* c = p + ((size_t)(g / kLane) * 16 + 15) * kLane + g % kLane;
    *c = EvolveConfidence(*c, tFrom, tTo, halfLife);
}

inline int32_t CenterInt(const hw_frame_interval& fi) { return fi.lower + (fi.upper - fi.lower) / 2; }

}   // namespace hwk

extern "C" int hw_detection_model_import(const hw_lane_model* d_models, uint32_t lanes, float* d_params, void* stream)
{
    using namespace hwk;
    if (!d_models || !d_params || lanes == 0) return SetLastError(HW_ERR_INVALID_ARG, "NULL argument or no lanes");
    ModelImportKernel<<<(lanes * kLane + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        d_models, d_params, (int)lanes);
    const cudaError_t ce = cudaGetLastError();
    return ce == cudaSuccess ? HW_OK : SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
}

extern "C" int hw_detection_model_export(const float* d_params, uint32_t lanes, hw_lane_model* d_models, void* stream)
{
    using namespace hwk;
    if (!d_models || !d_params || lanes == 0) return SetLastError(HW_ERR_INVALID_ARG, "NULL argument or no lanes");
    ModelExportKernel<<<(lanes * kLane + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        d_params, d_models, (int)lanes);
    const cudaError_t ce = cudaGetLastError();
    return ce == cudaSuccess ? HW_OK : SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
}

extern "C" int hw_detection_model_evolve_confidence(float* d_params, uint32_t lanes, hw_frame_interval from,
                                                    hw_frame_interval to, float half_life, void* stream)
{
    using namespace hwk;
    if (!d_params || lanes == 0) return SetLastError(HW_ERR_INVALID_ARG, "NULL argument or no lanes");
    if (from.lower >= from.upper || to.lower >= to.upper)
        return SetLastError(HW_ERR_INVALID_ARG, "frame intervals must not be empty");
    ModelEvolveKernel<<<(lanes * kLane + 127) / 128, 128, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
        d_params, (int)lanes, CenterInt(from), CenterInt(to), half_life);
    const cudaError_t ce = cudaGetLastError();
    return ce == cudaSuccess ? HW_OK : SetLastError(HW_ERR_CUDA, cudaGetErrorString(ce));
}
