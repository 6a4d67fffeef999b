// CPU oracle for the smrt-basecaller trace-analysis chain.
//
// TEST INFRASTRUCTURE ONLY.  This file restates, on the CPU, the reference's
// Host* implementations of the path (cdunn2001/hw, src/basecaller/...), so
// that tests can check the CUDA library against it and bench.py can time it
// as the CPU baseline.  Nothing in the hw_b200 product loads or calls it.
//
// The restatement is literal: every stage keeps the reference's order of
// floating-point operations, its lane-wide (64-ZMW) control flow, its integer
// wrap-around and its float->int conversions (cvtps2dq semantics).  exp/log
// are the project's Cephes-method routines (hw_b200/csrc/hw_math.h), the same
// ones the kernels call; the reference uses an SSE port of Cephes.  pow, exp2
// and log2 (used a few times per estimate) are evaluated in double precision
// and rounded to float on both sides.
//
// Each function cites the reference file:line it follows.  Abbreviations:
//   TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes,
//   CM = src/basecaller/common, AN = src/basecaller/basecaller/analyzer.
//
// Build: oracle/Makefile (g++ -O3 -march=native -ffp-contract=off -fopenmp).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <deque>
#include <limits>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include <omp.h>

#include "../include/hw_b200.h"
#include "../hw_b200/csrc/hw_math.h"
#include "../hw_b200/csrc/hw_params.h"

using namespace hwm;
using hwp::kLane;
using hwp::kAnalogs;
using hwp::kBins;
using hwp::kStates;

#define FZ for (int z = 0; z < kLane; ++z)

namespace {

thread_local std::string g_err;

const float kInf = std::numeric_limits<float>::infinity();
const float kNaN = std::numeric_limits<float>::quiet_NaN();

inline float pow_f(float x, float y) { return (float)std::pow((double)x, (double)y); }
inline float exp2_f(float x) { return (float)std::exp2((double)x); }
inline float log2_f(float x) { return (float)std::log2((double)x); }

// ---------------------------------------------------------------------------
// CM/StatAccumulator.h:48-252 (offset is always 0 on this path).
struct StatAcc
{
    float off[kLane], m0[kLane], m1[kLane], m2[kLane];
    void Reset() { FZ { off[z] = 0; m0[z] = 0; m1[z] = 0; m2[z] = 0; } }
    void Load(const hw_stat_accum_state& s)
    { FZ { off[z] = s.offset[z]; m0[z] = s.moment0[z]; m1[z] = s.moment1[z]; m2[z] = s.moment2[z]; } }
    void Store(hw_stat_accum_state& s) const
    { FZ { s.offset[z] = off[z]; s.moment0[z] = m0[z]; s.moment1[z] = m1[z]; s.moment2[z] = m2[z]; } }
    // AddSample(value), :160-166
    void Add(int z, float v) { const float x = v - off[z]; m0[z] += 1.0f; m1[z] += x; m2[z] += x * x; }
    // AddSample(value, mask), :168-174
    void AddMasked(int z, float v, bool m)
    {
        const float x = v - off[z];
        const float a0 = m0[z] + 1.0f, a1 = m1[z] + x, a2 = m2[z] + x * x;
        m0[z] = m ? a0 : m0[z]; m1[z] = m ? a1 : m1[z]; m2[z] = m ? a2 : m2[z];
    }
    // Merge, :176-184
    void Merge(const StatAcc& o) { FZ { m0[z] += o.m0[z]; m1[z] += o.m1[z]; m2[z] += o.m2[z]; } }
    // Mean, :85-88
    float Mean(int z) const { return m1[z] / m0[z] + off[z]; }
    // Variance, :90-97
    float Variance(int z) const
    {
        float var = m1[z] * m1[z] / m0[z];
        var = (m2[z] - var) / (m0[z] - 1.0f);
        var = fmax_sse(var, 0.0f);
        return (m0[z] > 1.0f) ? var : kNaN;
    }
};

// CM/AutocorrAccumulator.{h,cpp} with lag 4.
struct AutocorrAcc
{
    StatAcc stats;
    float m2[kLane];
    float fBuf[4][kLane], bBuf[4][kLane];
    uint16_t fbi, bbi;
    void Reset()
    {
        stats.Reset();
        FZ { m2[z] = 0; for (int k = 0; k < 4; ++k) { fBuf[k][z] = 0; bBuf[k][z] = 0; } }
        fbi = 0; bbi = 0;
    }
    void Load(const hw_autocorr_accum_state& s)
    {
        stats.Load(s.basic_stats);
        FZ { m2[z] = s.moment2[z]; for (int k = 0; k < 4; ++k) { fBuf[k][z] = s.fbuf[k][z]; bBuf[k][z] = s.bbuf[k][z]; } }
        fbi = s.bidx[0][0]; bbi = s.bidx[1][0];
    }
    void Store(hw_autocorr_accum_state& s) const
    {
        stats.Store(s.basic_stats);
        FZ { s.moment2[z] = m2[z]; for (int k = 0; k < 4; ++k) { s.fbuf[k][z] = fBuf[k][z]; s.bbuf[k][z] = bBuf[k][z]; } }
        FZ { s.bidx[0][z] = (uint8_t)fbi; s.bidx[1][z] = (uint8_t)bbi; }
    }
    // AddSample, AutocorrAccumulator.cpp:29-39 (lane-wide indices)
    void AddRow(const float* v)
    {
        const bool fill = fbi < 4;
        const int slot = bbi % 4;
        FZ
        {
            const float x = v[z] - stats.off[z];
            if (fill) fBuf[fbi][z] = x;
            m2[z] += bBuf[slot][z] * x;
            bBuf[slot][z] = x;
            stats.Add(z, v[z]);
        }
        if (fill) ++fbi;
        bbi = (uint16_t)((bbi + 1) % 4);
    }
    // Merge, AutocorrAccumulator.cpp:71-103
    void Merge(const AutocorrAcc& t)
    {
        stats.Merge(t.stats);
        FZ m2[z] += t.m2[z];
        const int n1 = 4 - t.fbi;
        for (int k = 0; k < 4 - n1; ++k)
        {
            const int i = (bbi + k) % 4, j = (t.bbi + n1 + k) % 4;
            FZ { m2[z] += bBuf[i][z] * t.fBuf[k][z]; bBuf[i][z] = t.bBuf[j][z]; }
        }
        const int n2 = 4 - fbi;
        for (int k = 0; k < n2; ++k) FZ fBuf[fbi + k][z] = t.fBuf[k][z];
        fbi = (uint16_t)(fbi + n2);
        bbi = (uint16_t)((bbi + (4 - n1)) % 4);
    }
};

// DT/BaselinerStatAccumulator.{h,cpp}
struct BlStatAcc
{
    AutocorrAcc corr;
    int16_t tmin[kLane], tmax[kLane];
    StatAcc blStats;
    float rawSum[kLane];
    StatAcc bgStats;
    void Reset()
    {
        corr.Reset(); blStats.Reset(); bgStats.Reset();
        FZ { tmin[z] = 32767; tmax[z] = -32768; rawSum[z] = 0.0f; }
    }
    void Load(const hw_baseliner_stats& s)
    {
        corr.Load(s.full_autocorr);
        FZ { tmin[z] = s.trace_min[z]; tmax[z] = s.trace_max[z]; rawSum[z] = s.raw_baseline_sum[z]; }
        blStats.Load(s.baseline_stats); bgStats.Load(s.background_stats);
    }
    void Store(hw_baseliner_stats& s) const
    {
        corr.Store(s.full_autocorr);
        FZ { s.trace_min[z] = tmin[z]; s.trace_max[z] = tmax[z]; s.raw_baseline_sum[z] = rawSum[z]; }
        blStats.Store(s.baseline_stats); bgStats.Store(s.background_stats);
    }
    // AddSample, BaselinerStatAccumulator.cpp:39-53
    void AddSample(const int16_t* raw, const int16_t* bls, const bool* isBl)
    {
        float bs[kLane];
        FZ bs[z] = (float)bls[z];
        corr.AddRow(bs);
        FZ
        {
            tmin[z] = std::min(bls[z], tmin[z]);
            tmax[z] = std::max(bls[z], tmax[z]);
            blStats.AddMasked(z, bs[z], isBl[z]);
            rawSum[z] += (float)(isBl[z] ? raw[z] : (int16_t)0);
        }
    }
    // Merge, BaselinerStatAccumulator.cpp:62-73
    void Merge(const BlStatAcc& o)
    {
        corr.Merge(o.corr);
        FZ { tmin[z] = std::min(tmin[z], o.tmin[z]); tmax[z] = std::max(tmax[z], o.tmax[z]); }
        blStats.Merge(o.blStats);
        FZ rawSum[z] += o.rawSum[z];
        bgStats.Merge(o.bgStats);
    }
};

// ---------------------------------------------------------------------------
// Baseliner: TA/HostMultiScaleBaseliner.{h,cpp}, TA/BlockFilterStage.cpp,
// TA/TraceFilters.cpp, TA/WindowBuffer.h.

// WindowBuffer<LaneArray<short>> with capacity w, always full after
// construction (w zeros pushed, BlockFilterStage.h:24-31).
struct WinBuf
{
    int w = 0, start = 0, counter = 0;
    std::vector<int16_t> d;      // w slots x 64
    int16_t hold[kLane];
    void Init(int width)
    {
        w = width; start = 0; counter = 0;
        d.assign((size_t)w * kLane, 0);
        FZ hold[z] = 0;
    }
    int16_t* at(int j) { return &d[(size_t)((start + j) % w) * kLane]; }
    void push(const int16_t* x)
    {
        std::memcpy(&d[(size_t)start * kLane], x, sizeof(int16_t) * kLane);
        start = (start + 1) % w;
        counter = (counter + 1) % w;
    }
};

struct Stage
{
    hwp::StageSpec spec;
    WinBuf wb;
    // BlockFilterStage::operator() + extremumFilterHgw (TraceFilters.cpp:11-57),
    // in place on block[F][64].
    void Run(int16_t* block, int F)
    {
        const int w = spec.width;
        const int dist = F / spec.nf;
        int16_t s[kLane], front[kLane], y[kLane];
        std::memcpy(s, wb.hold, sizeof(s));
        int outIdx = 0;
        auto op = [this](int16_t a, int16_t b) -> int16_t {
            return spec.isMax ? std::max(a, b) : std::min(a, b);
        };
        for (int i = 0; i < dist; i += spec.stride)
        {
            if (wb.counter == 0)
            {
                for (int j = w - 1; j > 0; --j)
                {
                    int16_t* rj = wb.at(j); int16_t* rj1 = wb.at(j - 1);
                    FZ rj1[z] = op(rj[z], rj1[z]);
                }
                std::memcpy(s, wb.at(w - 1), sizeof(s));
            }
            else
            {
                const int16_t* b = wb.at(w - 1);
                FZ s[z] = op(s[z], b[z]);
            }
            std::memcpy(front, wb.at(0), sizeof(front));
            wb.push(block + (size_t)i * kLane);
            FZ y[z] = op(s[z], front[z]);
            std::memcpy(block + (size_t)outIdx * kLane, y, sizeof(y));
            ++outIdx;
        }
        std::memcpy(wb.hold, s, sizeof(s));
    }
};

struct LaneBaseliner
{
    std::vector<Stage> lower, upper;
    float uemaSum[kLane], uemaWeight[kLane], sigmaEma[kLane];
    int16_t latData[kLane], latRaw[kLane];
    bool latL[kLane], latH1[kLane], latH2[kLane];

    void Init(const hwp::Derived& d)
    {
        hwp::StageSpec sp[2 * hwp::kMaxScales];
        int n = hwp::StageSpecs(d.fp, false, sp);
        lower.resize(n);
        for (int i = 0; i < n; ++i) { lower[i].spec = sp[i]; lower[i].wb.Init(sp[i].width); }
        n = hwp::StageSpecs(d.fp, true, sp);
        upper.resize(n);
        for (int i = 0; i < n; ++i) { upper[i].spec = sp[i]; upper[i].wb.Init(sp[i].width); }
        FZ
        {
            uemaSum[z] = 0.0f; uemaWeight[z] = 0.0f; sigmaEma[z] = 2.0f;
            latData[z] = 0; latRaw[z] = 0; latL[z] = latH1[z] = latH2[z] = false;
        }
    }

    // GetSmoothedBlEstimate, HostMultiScaleBaseliner.cpp:179-212
    void Smoothed(const hwp::Derived& d, const int16_t* lo, const int16_t* up, float* out)
    {
        constexpr float minSigma = .288675135f;
        const float ma = d.meanEmaAlpha, sa = d.sigmaEmaAlpha;
        FZ
        {
            const float sigma = fmax_sse((float)i16_wrap(up[z] - lo[z]) / d.cSigmaBias, minSigma);
            const float newSigmaEma = sa * sigmaEma[z] + (1.0f - sa) * sigma;
            const float blEst = 0.5f * (float)i16_wrap(up[z] + lo[z]) + d.cMeanBias * newSigmaEma;
            const bool mask = (uemaWeight[z] == 0.0f)
                            | (blEst - uemaSum[z] / uemaWeight[z] < d.jumpTolCoeff * sigmaEma[z]);
            const float newWeight = ma * uemaWeight[z] + (1.0f - ma);
            const float newSum = ma * uemaSum[z] + (1.0f - ma) * blEst;
            uemaWeight[z] = mask ? newWeight : uemaWeight[z];
            uemaSum[z] = mask ? newSum : uemaSum[z];
            sigmaEma[z] = mask ? newSigmaEma : sigmaEma[z];
            out[z] = uemaSum[z] / uemaWeight[z];
        }
    }

    // AddToBaselineStats, HostMultiScaleBaseliner.cpp:148-176
    void AddToStats(const hwp::Derived& d, const int16_t* trace, const int16_t* bls, BlStatAcc& st)
    {
        bool mask[kLane], hp1[kLane];
        FZ
        {
            const float thrLow = 4.5f * sigmaEma[z];
            const float thrHigh = 4.5f * sigmaEma[z];
            hp1[z] = (float)bls[z] < thrHigh * d.scaler;
            mask[z] = latH1[z] & latL[z] & hp1[z];
            latL[z] = (float)bls[z] < thrLow * d.scaler;
            latH2[z] = latH1[z];
            latH1[z] = hp1[z];
        }
        st.AddSample(latRaw, latData, mask);
        FZ { latRaw[z] = trace[z]; latData[z] = bls[z]; }
    }

    // EstimateBaseline, HostMultiScaleBaseliner.cpp:95-146
    void Estimate(const hwp::Derived& d, const int16_t* trace, int F, int16_t* out, BlStatAcc& st,
                  std::vector<int16_t>& lo, std::vector<int16_t>& up)
    {
        lo.assign(trace, trace + (size_t)F * kLane);
        up.assign(trace, trace + (size_t)F * kLane);
        for (auto& s : lower) s.Run(lo.data(), F);
        for (auto& s : upper) s.Run(up.data(), F);
        const int stride = d.aggStride;
        const int fdSize = F / stride;
        st.Reset();
        int t = 0;
        int16_t lv[kLane], uv[kLane], raw[kLane], bls[kLane], bg[kLane];
        float blEst[kLane], sub[kLane];
        for (int i = 0; i < fdSize; ++i)
        {
            FZ
            {
                lv[z] = i16_wrap(lo[(size_t)i * kLane + z] - d.pedestal);
                uv[z] = i16_wrap(up[(size_t)i * kLane + z] - d.pedestal);
            }
            Smoothed(d, lv, uv, blEst);
            FZ sub[z] = blEst[z] * d.scaler;
            for (int j = 0; j < stride; ++j, ++t)
            {
                const int16_t* tr = trace + (size_t)t * kLane;
                FZ
                {
                    const float rs = (float)i16_wrap(tr[z] - d.pedestal) * d.scaler;
                    bls[z] = to_i16_wrap(rs - sub[z]);
                    raw[z] = to_i16_wrap(rs);
                    out[(size_t)t * kLane + z] = bls[z];
                }
                AddToStats(d, raw, bls, st);
            }
            FZ bg[z] = to_i16_wrap(sub[z]);
            FZ st.bgStats.Add(z, (float)bg[z]);
        }
    }
};

// ---------------------------------------------------------------------------
// Histogram: TA/TraceHistogramAccumHost.cpp, TA/EdgeFrameClassifier.h,
// DT/UHistogramSimd.{h,cpp}

struct LaneHist
{
    float lower[kLane], binSize[kLane];
    uint16_t nLow[kLane], nHigh[kLane];
    uint16_t count[kBins + 1][kLane];
    bool valid = false;
};

struct EdgeClassifier
{
    int16_t prev[kLane];
    bool hist[2][kLane];
    int hsize;   // 0, 1, 2 (full)
    int hfront;
    void Init() { FZ { prev[z] = 0; hist[0][z] = hist[1][z] = false; } hsize = 0; hfront = 0; }
};

// UHistogramSimd ctor, UHistogramSimd.cpp:51-97: returns false on the
// reference's throw conditions.
bool HistInit(LaneHist& h, const float* lo, const float* up)
{
    bool ok = true;
    FZ
    {
        if (lo[z] >= up[z]) ok = false;
        const float bs = (up[z] - lo[z]) / static_cast<float>(kBins);
        if (bs <= 0.0f) ok = false;
        // binStart_[i] = binSize_*i + lowerBound must strictly change
        // (the last boundary is then overwritten by upperBound).
        float prevStart = lo[z];
        for (int i = 1; i <= kBins; ++i)
        {
            const float si = bs * (float)i + lo[z];
            if (prevStart == si) ok = false;
            prevStart = si;
        }
        h.lower[z] = lo[z];
        h.binSize[z] = bs;
        h.nLow[z] = 0; h.nHigh[z] = 0;
        for (int b = 0; b <= kBins; ++b) h.count[b][z] = 0;
    }
    h.valid = true;
    return ok;
}

// ---------------------------------------------------------------------------
// Detection model (float view): TA/DetectionModelHost.{h,cpp}

struct Model
{
    float bw[kLane], bm[kLane], bv[kLane];
    float aw[kAnalogs][kLane], am[kAnalogs][kLane], av[kAnalogs][kLane];
    float conf[kLane];
    hw_frame_interval fi;
};

inline int32_t CenterInt(const hw_frame_interval& fi) { return fi.lower + (fi.upper - fi.lower) / 2; }

void ModelFromLane(const hw_lane_model& l, hw_frame_interval fi, Model& m)
{
    FZ
    {
        m.bw[z] = f16_bits_to_f32(l.baseline.weights[z]);
        m.bm[z] = f16_bits_to_f32(l.baseline.means[z]);
        m.bv[z] = f16_bits_to_f32(l.baseline.vars[z]);
        for (int a = 0; a < kAnalogs; ++a)
        {
            m.aw[a][z] = f16_bits_to_f32(l.analogs[a].weights[z]);
            m.am[a][z] = f16_bits_to_f32(l.analogs[a].means[z]);
            m.av[a][z] = f16_bits_to_f32(l.analogs[a].vars[z]);
        }
        m.conf[z] = f16_bits_to_f32(l.confidence[z]);
    }
    m.fi = fi;
}

// EvolveConfidence, DetectionModelHost.h:189-201 (interval centres t0, t1)
void EvolveConfidence(Model& m, int32_t t0, int32_t t1, float halfLife)
{
    const float tDiff = static_cast<float>(t1 - t0);
    FZ { const float f = exp2_f(-std::abs(tDiff) / halfLife); m.conf[z] *= f; }
}

// ExportTo, DetectionModelHost.cpp:226-234, 277-285
void ModelToLane(const Model& m, hw_lane_model& l)
{
    const float varMax = round_f16(65000.0f);
    FZ
    {
        l.baseline.weights[z] = f32_to_f16_bits(m.bw[z]);
        l.baseline.means[z] = f32_to_f16_bits(m.bm[z]);
        l.baseline.vars[z] = f32_to_f16_bits(fmin_sse(m.bv[z], varMax));
        for (int a = 0; a < kAnalogs; ++a)
        {
            l.analogs[a].weights[z] = f32_to_f16_bits(m.aw[a][z]);
            l.analogs[a].means[z] = f32_to_f16_bits(m.am[a][z]);
            l.analogs[a].vars[z] = f32_to_f16_bits(fmin_sse(m.av[a][z], varMax));
        }
        l.confidence[z] = f32_to_f16_bits(m.conf[z]);
    }
}

struct DmeCtx
{
    const hw_config* cfg;
    const hwp::Derived* d;
};

// ModelSignalCovar, DetectionModelHost.cpp:237-245
inline float SignalCovar(const DmeCtx& c, float cv2, float mean, float blVar)
{
    float r = blVar;
    r += c.cfg->shot_var_coeff * mean;
    r += cv2 * (mean * mean);
    return r;
}

// XsnCoeffCVSq, DetectionModelHost.cpp:248-256
inline float XsnCoeffCVSq(const DmeCtx& c, float mean, float covar, float blVar)
{
    float r = covar - blVar;
    r -= mean * c.cfg->shot_var_coeff;
    r /= (mean * mean);
    return r;
}

// Update0/1/2, DetectionModelHost.cpp:52-187
void ModelUpdate(const DmeCtx& c, Model& t, const Model& o, const float* fraction)
{
    const uint32_t method = c.cfg->model_update_method;
    FZ
    {
        const float a = 1.0f - fraction[z];
        const float b = fraction[z];
        if (method == 0)
        {
            t.bm[z] = a * t.bm[z] + b * o.bm[z];
            t.bv[z] = a * t.bv[z] + b * o.bv[z];
            for (int i = 0; i < kAnalogs; ++i)
            {
                t.am[i][z] = a * t.am[i][z] + b * o.am[i][z];
                t.av[i][z] = a * t.av[i][z] + b * o.av[i][z];
            }
        }
        else
        {
            const float prevBlCovar = t.bv[z];
            const float bw = a * t.bw[z] + b * o.bw[z];
            t.bw[z] = bw;
            t.bm[z] = a * t.bm[z] + b * o.bm[z];
            const float bv = pow_f(t.bv[z], a) * pow_f(o.bv[z], b);
            t.bv[z] = bv;
            const float aw = 0.25f * (1.0f - bw);
            for (int i = 0; i < kAnalogs; ++i)
            {
                t.aw[i][z] = aw;
                float cv2;
                if (method == 1)
                {
                    const float cv = c.cfg->analogs[i].excess_noise_cv;
                    cv2 = cv * cv;
                }
                else
                {
                    const float tX = XsnCoeffCVSq(c, t.am[i][z], t.av[i][z], prevBlCovar);
                    const float oX = XsnCoeffCVSq(c, o.am[i][z], o.av[i][z], o.bv[z]);
                    cv2 = a * tX + b * oX;
                }
                const float am = pow_f(t.am[i][z], a) * pow_f(o.am[i][z], b);
                t.am[i][z] = am;
                t.av[i][z] = SignalCovar(c, cv2, am, bv);
            }
        }
    }
    t.fi = o.fi;
}

// Update(other), DetectionModelHost.cpp:207-223
void ModelUpdate(const DmeCtx& c, Model& t, const Model& o)
{
    float confSum[kLane], frac[kLane];
    FZ
    {
        confSum[z] = t.conf[z] + o.conf[z];
        frac[z] = (confSum[z] > 0.0f) ? o.conf[z] / confSum[z] : 0.0f;
    }
    ModelUpdate(c, t, o, frac);
    FZ t.conf[z] = confSum[z];
}

}   // namespace

// ---------------------------------------------------------------------------
// The pool object: one instance of every filter for one pool.

struct OraclePool
{
    hw_config cfg;
    hwp::Derived d;
    uint32_t poolId, lanes, F;

    // Baseliner
    std::vector<LaneBaseliner> bl;
    int32_t blNextFrame = 0;
    // Aggregator
    std::vector<BlStatAcc> agg;
    hw_frame_interval aggFi{0, 0};
    // Histogram
    std::vector<LaneHist> hist;
    std::vector<EdgeClassifier> edge;
    bool histInit = false;
    hw_frame_interval histFi{0, 0};
    // Labeler latent state (FrameLabelerHost.cpp:54-114)
    std::vector<hw_lane_model> latModel;
    std::vector<int16_t> latLabel, latRoi, latTrc, prevLat;   // [lane][64], [lane][24][64]
    // Pulse accumulator segments (HostPulseAccumulator.h:64-173)
    struct Segment
    {
        uint32_t start[kLane], end[kLane];
        int16_t first[kLane], last[kLane], mx[kLane];
        float total[kLane], m2[kLane];
        int16_t label[kLane];
    };
    std::vector<Segment> seg;

    bool Init(const hw_config& c, uint32_t pid, uint32_t nl, uint32_t f)
    {
        cfg = c; poolId = pid; lanes = nl; F = f;
        std::string err;
        if (!hwp::Validate(cfg, &err) || !hwp::Derive(cfg, &d, &err)) { g_err = err; return false; }
        if (F % d.aggStride != 0 || F < (uint32_t)hwp::kLatentFrames + hwp::kViterbiStitchLookback)
        { g_err = "frames_per_chunk incompatible with the filter strides or latency"; return false; }
        bl.resize(lanes);
        for (auto& b : bl) b.Init(d);
        agg.resize(lanes);
        for (auto& a : agg) a.Reset();
        hist.resize(lanes);
        edge.resize(lanes);
        for (auto& e : edge) e.Init();
        latModel.resize(lanes);
        latLabel.assign((size_t)lanes * kLane, 0);
        latRoi.assign((size_t)lanes * kLane, 0);
        latTrc.assign((size_t)lanes * kLane, 0);
        prevLat.assign((size_t)lanes * hwp::kLatentFrames * kLane, 0);
        for (auto& m : latModel)
        {
            std::memset(&m, 0, sizeof(m));
            FZ
            {
                m.baseline.means[z] = f32_to_f16_bits(0.0f);
                m.baseline.vars[z] = f32_to_f16_bits(50.0f);
                for (int a = 0; a < kAnalogs; ++a)
                {
                    m.analogs[a].means[z] = f32_to_f16_bits(1000.0f);
                    m.analogs[a].vars[z] = f32_to_f16_bits(10.0f);
                }
            }
        }
        seg.resize(lanes);
        for (auto& s : seg) std::memset(&s, 0, sizeof(s));
        return true;
    }

    // ---- Baseliner --------------------------------------------------------
    int Baseline(const int16_t* trace, int32_t firstFrame, int16_t* out, hw_baseliner_stats* stats)
    {
        const size_t blk = (size_t)F * kLane;
        int status = HW_OK;
#pragma omp parallel
        {
            std::vector<int16_t> lo, up;
            BlStatAcc st;
#pragma omp for schedule(dynamic, 4)
            for (int64_t l = 0; l < (int64_t)lanes; ++l)
            {
                bl[l].Estimate(d, trace + l * blk, (int)F, out + l * blk, st, lo, up);
                st.Store(stats[l]);
            }
        }
        blNextFrame = firstFrame + (int32_t)F;
        return status;
    }

    // ---- BaselineStatsAggregatorHost.cpp --------------------------------
    void AggAdd(const hw_baseliner_stats* stats, hw_frame_interval fi)
    {
#pragma omp parallel for schedule(static)
        for (int64_t l = 0; l < (int64_t)lanes; ++l)
        {
            BlStatAcc o;
            o.Load(stats[l]);
            agg[l].Merge(o);
        }
        if (aggFi.lower == aggFi.upper) aggFi = fi;
        else if (fi.lower != fi.upper)
            aggFi = hw_frame_interval{std::min(aggFi.lower, fi.lower), std::max(aggFi.upper, fi.upper)};
    }
    void AggGet(hw_baseliner_stats* out, hw_frame_interval* fi) const
    {
        for (uint32_t l = 0; l < lanes; ++l) agg[l].Store(out[l]);
        if (fi) *fi = aggFi;
    }
    void AggReset()
    {
        for (auto& a : agg) a.Reset();
        aggFi = hw_frame_interval{0, 0};
    }

    // ---- TraceHistogramAccumHost::ResetImpl(metrics), :96-126 -----------
    int HistResetStats(const hw_baseliner_stats* stats)
    {
        bool ok = true;
        for (uint32_t l = 0; l < lanes; ++l)
        {
            StatAcc s;
            s.Load(stats[l].baseline_stats);
            float lo[kLane], up[kLane];
            FZ
            {
                const bool suff = s.m0[z] >= (float)cfg.baseline_stat_min_frame_count;
                const float mean = suff ? s.Mean(z) : 0.0f;
                const float sigma = suff ? std::sqrt(s.Variance(z)) : cfg.fallback_baseline_sigma;
                const float binSize = fmax_sse(cfg.bin_size_coeff * sigma, d.binSizeMin);
                lo[z] = mean - 4.0f * sigma;
                up[z] = lo[z] + float(kBins) * binSize;
            }
            ok &= HistInit(hist[l], lo, up);
        }
        histInit = true;
        histFi = hw_frame_interval{0, 0};
        if (!ok) { g_err = "UHistogramSimd: bad histogram bounds"; return HW_ERR_NUMERIC; }
        return HW_OK;
    }

    int HistResetBounds(const hw_lane_hist_bounds* b)
    {
        bool ok = true;
        for (uint32_t l = 0; l < lanes; ++l) ok &= HistInit(hist[l], b[l].lower_bounds, b[l].upper_bounds);
        histInit = true;
        histFi = hw_frame_interval{0, 0};
        if (!ok) { g_err = "UHistogramSimd: bad histogram bounds"; return HW_ERR_NUMERIC; }
        return HW_OK;
    }

    // ---- AddBlock, TraceHistogramAccumHost.cpp:140-169 ------------------
    int HistAdd(const int16_t* traces, uint32_t frames, hw_frame_interval fi, const hw_lane_model* models)
    {
        if (!histInit)
        {
            g_err = "Cannot aggregate trace data into histograms before calling Reset with the desired histogram bounds";
            return HW_ERR_NOT_INITIALIZED;
        }
#pragma omp parallel for schedule(dynamic, 4)
        for (int64_t l = 0; l < (int64_t)lanes; ++l)
        {
            LaneHist& h = hist[l];
            EdgeClassifier& e = edge[l];
            int16_t thr[kLane];
            FZ
            {
                const float bm = f16_bits_to_f32(models[l].baseline.means[z]);
                const float bv = f16_bits_to_f32(models[l].baseline.vars[z]);
                thr[z] = i16_wrap(cvt_rn_i32(2.0f * std::sqrt(bv) + bm));
            }
            const int16_t* tr = traces + (size_t)l * frames * kLane;
            for (uint32_t f = 0; f < frames; ++f)
            {
                const int16_t* fr = tr + (size_t)f * kLane;
                const bool full = (e.hsize == 2);
                const int slotFront = e.hfront;
                FZ
                {
                    // EdgeFrameClassifier::IsEdgeFrame (EdgeFrameClassifier.h:72-94)
                    const bool isBl = fr[z] < thr[z];
                    const bool edgeF = full ? (isBl ^ e.hist[slotFront][z]) : true;
                    const int16_t cand = e.prev[z];
                    e.prev[z] = fr[z];
                    // UHistogramSimd::AddDatum (UHistogramSimd.h:207-229)
                    const bool sel = !edgeF;
                    const float x = (float)cand;
                    int32_t bin = floor_cast_i32((x - h.lower[z]) / h.binSize[z]);
                    const bool mLow = sel & (bin < 0);
                    const bool mHigh = sel & (bin >= kBins);
                    if (mLow) h.nLow[z] = (uint16_t)(h.nLow[z] + 1);
                    if (mHigh) h.nHigh[z] = (uint16_t)(h.nHigh[z] + 1);
                    if ((!sel) | mLow | mHigh) bin = kBins;
                    h.count[bin][z] = (uint16_t)(h.count[bin][z] + 1);
                }
                // CircularArray<LaneMask,2>::push_back (CM/CircularArray.h)
                if (e.hsize < 2)
                {
                    const int slot = (e.hfront + e.hsize) % 2;
                    FZ e.hist[slot][z] = fr[z] < thr[z];
                    ++e.hsize;
                }
                else
                {
                    const int slot = e.hfront;
                    FZ e.hist[slot][z] = fr[z] < thr[z];
                    e.hfront = (e.hfront + 1) % 2;
                }
            }
        }
        if (histFi.lower == histFi.upper) histFi = fi;
        else histFi = hw_frame_interval{std::min(histFi.lower, fi.lower), std::max(histFi.upper, fi.upper)};
        return HW_OK;
    }

    // HistogramImpl, TraceHistogramAccumHost.cpp:172-199
    void HistGet(hw_lane_histogram* out, hw_frame_interval* fi) const
    {
        for (uint32_t l = 0; l < lanes; ++l)
        {
            const LaneHist& h = hist[l];
            FZ
            {
                out[l].low_bound[z] = h.lower[z];
                out[l].bin_size[z] = h.binSize[z];
                out[l].outlier_count_low[z] = h.nLow[z];
                out[l].outlier_count_high[z] = h.nHigh[z];
                for (int b = 0; b < kBins; ++b) out[l].bin_count[b][z] = h.count[b][z];
            }
        }
        if (fi) *fi = histFi;
    }

    // ---- DmeEmHost::InitLaneDetModel, DmeEmHost.cpp:872-925 -------------
    void InitModels(const hw_baseliner_stats* stats, hw_lane_model* out)
    {
        const DmeCtx c{&cfg, &d};
        const bool fixedBl = false;
        for (uint32_t l = 0; l < lanes; ++l)
        {
            StatAcc blS, tot;
            blS.Load(stats[l].baseline_stats);
            tot.Load(stats[l].full_autocorr.basic_stats);
            hw_lane_model& m = out[l];
            FZ
            {
                const float blWeight = blS.m0[z] / tot.m0[z];
                float blMean = fixedBl ? 0.0f : blS.Mean(z);
                float blVar = blS.Variance(z);
                blMean = std::isnan(blMean) ? 0.0f : blMean;     // FallbackBaselineMean
                blVar = std::isnan(blVar) ? 100.0f : blVar;      // FallbackBaselineVariance
                blVar = fmin_sse(fmax_sse(blVar, d.blVarMin), d.blVarMax);
                m.confidence[z] = f32_to_f16_bits(0.1f);
                m.baseline.weights[z] = f32_to_f16_bits(blWeight);
                m.baseline.means[z] = f32_to_f16_bits(blMean);
                m.baseline.vars[z] = f32_to_f16_bits(blVar);
                const float amw = (1.0f - blWeight) / (float)kAnalogs;
                const float refSignal = cfg.ref_snr * std::sqrt(blVar);
                for (int a = 0; a < kAnalogs; ++a)
                {
                    m.analogs[a].weights[z] = f32_to_f16_bits(amw);
                    const float aMean = fmax_sse(0.0f, blMean + cfg.analogs[a].rel_amplitude * refSignal);
                    m.analogs[a].means[z] = f32_to_f16_bits(aMean);
                    const float cv = cfg.analogs[a].excess_noise_cv;
                    m.analogs[a].vars[z] = f32_to_f16_bits(SignalCovar(c, cv * cv, aMean, blVar));
                }
            }
        }
    }

    int Estimate(const hw_lane_histogram* h, const hw_baseliner_stats* stats, hw_frame_interval histFi_,
                 hw_frame_interval modelFi, hw_lane_model* models, hw_dme_diag* diag,
                 const float* proposal = nullptr);

    // The DME's work before its EM iterations, for lane l (see the definition).
    using LaneEmRef = void*;
    void DmePrelude(int64_t l, const hw_lane_histogram* hh, const hw_baseliner_stats* stats,
                    hw_frame_interval hfi, hw_frame_interval pfi, const hw_lane_model* models, Model& det,
                    LaneEmRef em);

    int EmFit(const hw_lane_histogram* hh, const hw_baseliner_stats* stats, hw_frame_interval hfi,
              hw_frame_interval pfi, const hw_lane_model* models, int mode, const float* proposal,
              const float* target, float tol, uint32_t maxIter, float* params, int32_t* iters, float* loglike,
              float* atStop);

    int Label(const int16_t* traces, const hw_lane_model* models, int16_t* labels, int16_t* latOut, float* score,
              float* margin);

    int Pulses(const int16_t* labels, const int16_t* latTrace, const int16_t* trace, int32_t firstFrame,
               const hw_lane_model* models, hw_pulse* pulses, uint32_t* lens, uint32_t* ovf,
               hw_stat_accum_state* blstats);
};

// ---------------------------------------------------------------------------
// DME: TA/DmeEmHost.cpp:131-852

namespace {

struct UHist   // UHistogramSimd built from a LaneHistogram (UHistogramSimd.cpp:100-121)
{
    const hw_lane_histogram* h;
    float BinStart(int b, int z) const { return h->low_bound[z] + (float)b * h->bin_size[z]; }
    uint16_t Count(int b, int z) const { return b < kBins ? h->bin_count[b][z] : (uint16_t)0; }
    uint16_t InRange(int z) const
    {
        uint16_t s = 0;
        for (int b = 0; b < kBins; ++b) s = (uint16_t)(s + h->bin_count[b][z]);
        return s;
    }
    uint16_t Total(int z) const
    { return (uint16_t)(InRange(z) + (uint16_t)(h->outlier_count_low[z] + h->outlier_count_high[z])); }

    // CumulativeCount, UHistogramSimd.cpp:204-242
    float Cumulative(float x, int z) const
    {
        const float lb = BinStart(0, z), ub = BinStart(kBins, z);
        const bool mNan = std::isnan(x), mLow = x < lb, mHigh = x >= ub;
        const bool inB = !(mNan | mLow | mHigh);
        int32_t xbin = floor_cast_i32((x - lb) / h->bin_size[z]);
        xbin = inB ? xbin : 0;
        const float xrem = x - BinStart(xbin, z);
        const float xbinCount = (float)Count(xbin, z);
        float cc = (float)h->outlier_count_low[z];
        uint16_t cn = 0;
        for (int i = 0; i < std::min(kBins, xbin); ++i) cn = (uint16_t)(cn + h->bin_count[i][z]);
        cc += (float)cn;
        cc += xbinCount * xrem / h->bin_size[z];
        cc = mLow ? (float)h->outlier_count_low[z] : cc;
        cc = mHigh ? (float)(uint16_t)(h->outlier_count_low[z] + InRange(z)) : cc;
        cc = mNan ? kNaN : cc;
        return cc;
    }

    // Fractile, UHistogramSimd.cpp:142-201 (per ZMW)
    float Fractile(float frac, int z) const
    {
        const float nfz = frac * (float)Total(z);
        uint16_t n = h->outlier_count_low[z];
        if (n > 0 && n >= nfz) return -kInf;
        int i = 0;
        while ((n == 0 || n < nfz) && i < kBins) n = (uint16_t)(n + h->bin_count[i++][z]);
        if (n < nfz) return kInf;
        i -= 1;
        const float x0 = BinStart(i, z);
        const uint16_t niz = h->bin_count[i][z];
        const int m = (int)n - (int)niz;
        return x0 + h->bin_size[z] * (nfz - (float)m) / (float)(niz + 1);
    }
};

}   // namespace

namespace {

// One lane's EM state and per-bin work arrays (DmeEmHost.cpp:253-565), with
// the E-step (cornerComp / centerComp over the 301 bin boundaries) and the
// M-step as methods so that the reference estimate and the single-ZMW fit of
// the learned initializer share the arithmetic.
struct LaneEm
{
    const DmeCtx& c;
    const hw_lane_histogram& hh;
    UHist hist;
    float* tau;        // [5][nB + 1][64]
    float* bprob;      // [nB + 1][64]
    float* binProb;    // [nB][64]
    float* nj;         // [nB][64]
    float rho[5][kLane], mu[5][kLane], var[5][kLane], s[kLane];
    float sExpect[kLane], sExpectW[kLane], varQuant[kLane], binProbMin[kLane], nSum[kLane];
    float varinv[5][kLane], ci[5][kLane], mom1[5][kLane];
    float rpa[kAnalogs];

    LaneEm(const DmeCtx& ctx, const hw_lane_histogram& h, float* t, float* bp, float* bpr, float* n)
        : c(ctx), hh(h), hist{&h}, tau(t), bprob(bp), binProb(bpr), nj(n)
    {
        for (int a = 0; a < kAnalogs; ++a) rpa[a] = c.cfg->analogs[a].rel_amplitude;
        FZ nSum[z] = 0.0f;
        for (int j = 0; j < kBins; ++j)
            FZ { nj[(size_t)j * kLane + z] = (float)hh.bin_count[j][z]; nSum[z] += nj[(size_t)j * kLane + z]; }
    }
    float* TAU(int m, int b) { return &tau[((size_t)m * (kBins + 1) + b) * kLane]; }
    float* BP(int b) { return &bprob[(size_t)b * kLane]; }
    float* BPR(int b) { return &binProb[(size_t)b * kLane]; }

    // s of the EM set-up from the current analog means (fixed-size-4 Eigen sum)
    void SetScale()
    {
        FZ
        {
            const float p0 = mu[1][z] * rpa[0], p1 = mu[2][z] * rpa[1], p2 = mu[3][z] * rpa[2], p3 = mu[4][z] * rpa[3];
            s[z] = ((p0 + p1) + (p2 + p3)) / c.d->rpaSum2;
        }
    }

    // E-step: log-likelihood per ZMW into ll, ci and mom1 filled.
    void EStep(float* ll)
    {
        const float halfLog2pi = 0.5f * c.d->logTwoPi;
        FZ for (int k = 0; k < 5; ++k)
        {
            varinv[k][z] = 1.0f / var[k][z];
            pref_[k][z] = (hw_logf(rho[k][z]) - 0.5f * hw_logf(var[k][z])) - halfLog2pi;
        }
        float probSum[kLane], wps[kLane];
        FZ { probSum[z] = 0; wps[z] = 0; for (int k = 0; k < 5; ++k) { ci[k][z] = 0; mom1[k][z] = 0; } }
        auto corner = [&](int b) {
            FZ
            {
                const float x = hist.BinStart(b, z);
                float t[5];
                for (int i = 0; i < 5; ++i)
                {
                    const float y = x - mu[i][z];
                    t[i] = pref_[i][z] - 0.5f * y * y * varinv[i][z];
                }
                float tmax = t[0];
                for (int i = 1; i < 5; ++i) tmax = fmax_sse(tmax, t[i]);
                float se = hw_expf(t[0] - tmax);
                for (int i = 1; i < 5; ++i) se = se + hw_expf(t[i] - tmax);
                const float llb = tmax + hw_logf(se);
                for (int i = 0; i < 5; ++i) TAU(i, b)[z] = hw_expf(t[i] - llb);
                BP(b)[z] = hw_expf(llb);
            }
        };
        auto center = [&](int b) {
            FZ
            {
                const float bs = hh.bin_size[z];
                const float bp0 = BP(b)[z], bp1 = BP(b + 1)[z];
                const float bpr = fmax_sse(0.5f * bs * (bp0 + bp1), binProbMin[z]);
                BPR(b)[z] = bpr;
                probSum[z] += bpr;
                const float njb = nj[(size_t)b * kLane + z];
                wps[z] += njb * hw_logf(bpr);
                const float factor = njb / bpr;
                const float x0 = hist.BinStart(b, z), x1 = hist.BinStart(b + 1, z);
                for (int m = 0; m < 5; ++m)
                {
                    const float tmp1 = bp0 * TAU(m, b)[z];
                    const float tmp2 = bp1 * TAU(m, b + 1)[z];
                    ci[m][z] += (tmp1 + tmp2) * factor;
                    mom1[m][z] += (tmp1 * x0 + tmp2 * x1) * factor;
                }
            }
        };
        corner(0);
        for (int b = 0; b < kBins; ++b) { corner(b + 1); center(b); }
        FZ
        {
            const float hb = 0.5f * hh.bin_size[z];
            for (int k = 0; k < 5; ++k) { ci[k][z] *= hb; mom1[k][z] *= hb; }
            float l = wps[z] - nSum[z] * hw_logf(probSum[z]);
            const float ds = s[z] - sExpect[z];
            l -= 0.5f * (ds * ds) * sExpectW[z];
            ll[z] = l;
        }
    }

    // M-step, DmeEmHost.cpp:494-565
    void MStep(int32_t* zStatus)
    {
        const hwp::Derived& d = *c.d;
        FZ
        {
            for (int k = 0; k < 5; ++k) ci[k][z] = fmax_sse(ci[k][z], 0.1f);
            for (int k = 0; k < 5; ++k) rho[k][z] = ci[k][z] / nSum[z];
            const float rs = (rho[0][z] + rho[1][z]) + (rho[2][z] + (rho[3][z] + rho[4][z]));
            for (int k = 0; k < 5; ++k) rho[k][z] = rho[k][z] / rs;
            mu[0][z] = mom1[0][z] / ci[0][z];
            float numer = 0.0f, denom = 0.0f;
            for (int a = 0; a < kAnalogs; ++a)
            {
                const int i = a + 1;
                numer += rpa[a] * varinv[i][z] * mom1[i][z];
                denom += (rpa[a] * rpa[a]) * varinv[i][z] * ci[i][z];
            }
            numer += sExpect[z] * sExpectW[z];
            denom += sExpectW[z];
            float sv = numer / denom;
            const float sMin = fmax_sse(0.5f * std::sqrt(var[0][z]), d.minPulseMean) / d.rpaMin;
            const bool vls = sv < sMin;
            sv = vls ? sMin : sv;
            if (vls) zStatus[z] |= 4;   // VLOW_SIGNAL
            s[z] = sv;
            for (int a = 0; a < kAnalogs; ++a) mu[a + 1][z] = sv * rpa[a];
        }
        float mom2[kLane];
        FZ mom2[z] = 0.0f;
        for (int j = 0; j < kBins; ++j)
        {
            const int k = j + 1;
            FZ
            {
                const float x0 = hist.BinStart(j, z) - mu[0][z];
                const float x1 = hist.BinStart(k, z) - mu[0][z];
                float tmp = BP(j)[z] * x0 * x0 * TAU(0, j)[z];
                tmp += BP(k)[z] * x1 * x1 * TAU(0, k)[z];
                tmp *= nj[(size_t)j * kLane + z] / BPR(j)[z];
                mom2[z] += tmp;
            }
        }
        FZ
        {
            mom2[z] *= 0.5f * hh.bin_size[z];
            float v0 = mom2[z] / ci[0][z] + varQuant[z];
            v0 = fmin_sse(fmax_sse(v0, d.blVarMin), d.blVarMax);
            var[0][z] = v0;
            for (int a = 0; a < kAnalogs; ++a)
            {
                const float cv = c.cfg->analogs[a].excess_noise_cv;
                var[a + 1][z] = SignalCovar(c, cv * cv, mu[a + 1][z], v0);
            }
        }
    }

    // The learned start: per ZMW, the proposal Q [15][64] replaces the current
    // (reference) start unless `fallback` is set and the proposal's
    // log-likelihood is lower (or not comparable).
    void ChooseStart(const float* Q, bool fallback, int32_t* fellBack, float* llPlain, float* llStart)
    {
        float rho0[5][kLane], mu0[5][kLane], var0[5][kLane], s0[kLane], llProp[kLane];
        EStep(llPlain);
        std::memcpy(rho0, rho, sizeof(rho0));
        std::memcpy(mu0, mu, sizeof(mu0));
        std::memcpy(var0, var, sizeof(var0));
        std::memcpy(s0, s, sizeof(s0));
        FZ for (int k = 0; k < 5; ++k)
        {
            rho[k][z] = Q[k * kLane + z];
            mu[k][z] = Q[(5 + k) * kLane + z];
            var[k][z] = Q[(10 + k) * kLane + z];
        }
        SetScale();
        EStep(llProp);
        FZ
        {
            fellBack[z] = 0;
            llStart[z] = llProp[z];
            if (fallback && !(llProp[z] >= llPlain[z]))
            {
                for (int k = 0; k < 5; ++k) { rho[k][z] = rho0[k][z]; mu[k][z] = mu0[k][z]; var[k][z] = var0[k][z]; }
                s[z] = s0[z];
                fellBack[z] = 1;
                llStart[z] = llPlain[z];
            }
        }
    }

private:
    float pref_[5][kLane];
};

}   // namespace

// EvolveModel, PrelimEstimate with its confidence-weighted update,
// PrelimScaleFactor, ScaleModelSnr and the EM set-up (DmeEmHost.cpp:161-361,
// 620-654, 806-852) for lane l: the updated prior model in det and the plain
// EM start in em.
void OraclePool::DmePrelude(int64_t l, const hw_lane_histogram* hh, const hw_baseliner_stats* stats,
                            hw_frame_interval hfi, hw_frame_interval pfi, const hw_lane_model* models, Model& det,
                            LaneEmRef emRef)
{
    LaneEm& em = *static_cast<LaneEm*>(emRef);
    const DmeCtx c{&cfg, &d};
    ModelFromLane(models[l], pfi, det);
    BlStatAcc bsa;
    bsa.Load(stats[l]);
    UHist hist{&hh[l]};

    // EvolveModel, DmeEmHost.cpp:806-834
    {
        const int32_t tModel = CenterInt(det.fi), tEst = CenterInt(hfi);
        const float thl = 0.5f * (float)(tModel + tEst);
        const float t0 = 56160.0f, t1 = 168480.0f;
        const float hl0 = cfg.confidence_half_life[0], hl1 = cfg.confidence_half_life[1];
        const float hl = hl0 + (hl1 - hl0) * satlin_std(t0, t1, thl);
        // EvolveConfidence, DetectionModelHost.h:166-177
        EvolveConfidence(det, CenterInt(det.fi), CenterInt(hfi), hl);
        det.fi = hfi;
    }

    // PrelimEstimate, DmeEmHost.cpp:161-214
    Model work = det;
    {
        const float blVarMax = d.blVarMax;
        FZ
        {
            const float nBl = bsa.blStats.m0[z];
            const float tot = bsa.corr.stats.m0[z];
            const float blWeight = fmax_sse(nBl / tot, 0.01f);
            const bool mask = nBl >= 3.0f;
            float blVar = mask ? bsa.blStats.Variance(z) : work.bv[z];
            blVar = fmin_sse(fmax_sse(blVar, d.blVarMin), blVarMax);
            const float blMean = mask ? bsa.blStats.Mean(z) : work.bm[z];
            const float scale = std::sqrt(blVar / work.bv[z]);
            for (int i = 0; i < kAnalogs; ++i)
            {
                const float mean = work.am[i][z] * scale;
                const float cv = cfg.analogs[i].excess_noise_cv;
                const float cv2 = cv * cv;
                work.am[i][z] = mean;
                work.av[i][z] = SignalCovar(c, cv2, mean, blVar);
                work.aw[i][z] = 0.25f * (1.0f - blWeight);
            }
            work.bw[z] = blWeight;
            work.bm[z] = blMean;
            work.bv[z] = blVar;
            float conf = 0.1f * satlin_sse(0.0f, 500.0f, nBl - 3.0f);
            conf *= satlin_sse(blVarMax, 0.5f * (d.blVarNominal + blVarMax), blVar);
            work.conf[z] = conf;
        }
    }
    ModelUpdate(c, det, work);
    work = det;

    // PrelimScaleFactor, DmeEmHost.cpp:620-654
    float scaleFactor[kLane];
    FZ
    {
        const float bgSigma = std::sqrt(work.bv[z]);
        const float thresh = 2.5f * bgSigma + work.bm[z];
        const float bgCount = hist.Cumulative(thresh, z);
        const float totalCount = (float)(uint16_t)(hh[l].outlier_count_low[z] + hist.InRange(z));
        const float fractile = 0.5f * (bgCount + totalCount) / totalCount;
        float avg = 0.0f;
        for (int a = 0; a < kAnalogs; ++a) avg += work.am[a][z];
        avg /= static_cast<float>(kAnalogs);
        const float w = satlin_sse(0.0f, cfg.scale_snr_conf_tol, work.conf[z]);
        float sf = hist.Fractile(fractile, z) / avg;
        sf = (1.0f - w) * sf + w;
        scaleFactor[z] = fmin_sse(fmax_sse(sf, 0.1f), 10.0f);
    }
    // ScaleModelSnr, DmeEmHost.cpp:837-852
    FZ
    {
        const float blCovar = work.bv[z];
        for (int a = 0; a < kAnalogs; ++a)
        {
            work.am[a][z] = scaleFactor[z] * work.am[a][z];
            const float cv = cfg.analogs[a].excess_noise_cv;
            work.av[a][z] = SignalCovar(c, cv * cv, work.am[a][z], blCovar);
        }
    }

    // EM setup, DmeEmHost.cpp:253-361
    const float rhoMin = 0.001f;
    FZ
    {
        em.rho[0][z] = fmax_sse(work.bw[z], rhoMin);
        em.mu[0][z] = work.bm[z];
        em.var[0][z] = work.bv[z];
        for (int a = 0; a < kAnalogs; ++a)
        {
            em.rho[a + 1][z] = fmax_sse(work.aw[a][z], rhoMin);
            em.mu[a + 1][z] = work.am[a][z];
            em.var[a + 1][z] = work.av[a][z];
        }
        const float bs = hh[l].bin_size[z];
        em.varQuant[z] = (bs * bs) / 12.0f;
        for (int k = 0; k < 5; ++k) em.var[k][z] += em.varQuant[z];
        em.var[0][z] = fmin_sse(em.var[0][z], d.blVarMax);
        // Eigen fixed-size-5 sum: (r0 + r1) + (r2 + (r3 + r4))
        const float rs = (em.rho[0][z] + em.rho[1][z]) + (em.rho[2][z] + (em.rho[3][z] + em.rho[4][z]));
        for (int k = 0; k < 5; ++k) em.rho[k][z] = em.rho[k][z] / rs;
        const uint16_t nf = hist.Total(z);
        em.binProbMin[z] = fmax_sse((float)nf * bs, 1.0f) * std::numeric_limits<float>::min();
    }
    em.SetScale();
    FZ
    {
        em.sExpect[z] = em.s[z] / scaleFactor[z];
        em.sExpectW[z] = det.conf[z] * cfg.pulse_amp_regularization;
    }
}

int OraclePool::Estimate(const hw_lane_histogram* hh, const hw_baseliner_stats* stats, hw_frame_interval hfi,
                         hw_frame_interval pfi, hw_lane_model* models, hw_dme_diag* diag, const float* proposal)
{
    const DmeCtx c{&cfg, &d};
    int status = HW_OK;
    std::string errMsg;
    const int nModes = kAnalogs + 1;
    const int nB = kBins;

#pragma omp parallel
    {
        std::vector<float> tau((size_t)nModes * (nB + 1) * kLane);
        std::vector<float> bprob((size_t)(nB + 1) * kLane), binProb((size_t)nB * kLane), nj((size_t)nB * kLane);
#pragma omp for schedule(dynamic, 1)
        for (int64_t l = 0; l < (int64_t)lanes; ++l)
        {
            auto emPtr = std::make_unique<LaneEm>(c, hh[l], tau.data(), bprob.data(), binProb.data(), nj.data());
            LaneEm& em = *emPtr;
            Model det;
            DmePrelude(l, hh, stats, hfi, pfi, models, det, &em);
            if (proposal)
            {
                int32_t fb[kLane];
                float l0[kLane], l1[kLane];
                em.ChooseStart(proposal + (size_t)l * 15 * kLane, true, fb, l0, l1);
            }
            UHist hist{&hh[l]};
            Model work;
            work.fi = hfi;

            float rhoEst[5][kLane], muEst[5][kLane], varEst[5][kLane];
            float logLike[kLane], ll[kLane];
            int32_t zStatus[kLane];
            bool conv[kLane], mConverged[kLane];
            int32_t mIter[kLane];
            float mLogLike[kLane];
            FZ
            {
                for (int k = 0; k < 5; ++k) { rhoEst[k][z] = em.rho[k][z]; muEst[k][z] = em.mu[k][z]; varEst[k][z] = em.var[k][z]; }
                logLike[z] = std::numeric_limits<float>::lowest();
                zStatus[z] = (hist.Total(z) < 160u) ? 2 /*INSUF_DATA*/ : 0;
                mConverged[z] = false; mIter[z] = 0; mLogLike[z] = -kInf;
            }

            const unsigned iterLimit = cfg.em_iteration_limit;
            unsigned it = 0;
            for (; it < iterLimit; ++it)
            {
                em.EStep(ll);
                bool anyConv = false, allDone = true;
                FZ
                {
                    const float prev = logLike[z];
                    logLike[z] = ll[z];
                    const float delta = ll[z] - prev;
                    const float convTol = 1e-4f * fmax_sse(ll[z], -ll[z]);
                    bool cv = (delta >= 0) & (delta < convTol);
                    cv &= (ll[z] >= mLogLike[z]);
                    conv[z] = cv;
                    // MaxLikelihoodDiagnostics::Converged (MaxLikelihoodDiagnostics.h:85-96)
                    mIter[z] = (cv & !mConverged[z]) ? (int32_t)it : mIter[z];
                    mLogLike[z] = cv ? ll[z] : mLogLike[z];
                    mConverged[z] |= cv;
                    anyConv |= cv;
                    allDone &= (mConverged[z] | (zStatus[z] != 0));
                }
                if (anyConv)
                    FZ for (int k = 0; k < 5; ++k)
                    {
                        rhoEst[k][z] = conv[z] ? em.rho[k][z] : rhoEst[k][z];
                        muEst[k][z] = conv[z] ? em.mu[k][z] : muEst[k][z];
                        varEst[k][z] = conv[z] ? em.var[k][z] : varEst[k][z];
                    }
                if (!cfg.iterate_to_limit && allDone) break;
                em.MStep(zStatus);
            }
            const int laneIters = (int)std::min(it + 1, iterLimit);

            bool finite = true;
            FZ
            {
                if (!mConverged[z]) zStatus[z] |= 1;    // NO_CONVERGE
                for (int k = 0; k < 5; ++k)
                    finite &= std::isfinite(rhoEst[k][z]) & std::isfinite(muEst[k][z]) & std::isfinite(varEst[k][z]);
                work.bw[z] = rhoEst[0][z]; work.bm[z] = muEst[0][z]; work.bv[z] = varEst[0][z];
                for (int a = 0; a < kAnalogs; ++a)
                { work.aw[a][z] = rhoEst[a + 1][z]; work.am[a][z] = muEst[a + 1][z]; work.av[a][z] = varEst[a + 1][z]; }
            }
            if (!finite)
            {
#pragma omp critical
                { status = HW_ERR_NUMERIC; errMsg = "DME: non-finite EM estimate (all(isfinite(...)) assertion)"; }
            }

            // ComputeConfidence, DmeEmHost.cpp:717-803 (G-test disabled: pValue = 1)
            float conf[kLane];
            bool assertOk = true;
            FZ
            {
                float cf[8];
                cf[0] = mConverged[z] ? 1.0f : 0.0f;
                cf[1] = satlin_sse(0.05f, 0.15f, work.bw[z]);
                float x = (work.bm[z] * work.bm[z]) / work.bv[z];
                x = hw_expf(-x / 2.0f);
                cf[2] = x;
                x = log2_f(work.bv[z] / det.bv[z]);
                const float bgVarTol = 1.5f / (0.5f + det.conf[z]);
                x = hw_expf(-x * x / (2.0f * (bgVarTol * bgVarTol)));
                cf[3] = x;
                x = 1.0f;
                if (cfg.analog_mix_fraction_threshold[1] > 0.0f)
                {
                    const float t0 = cfg.analog_mix_fraction_threshold[0], t1 = cfg.analog_mix_fraction_threshold[1];
                    x *= satlin_sse(t0, t1, work.aw[0][z]);
                    x *= satlin_sse(t0, t1, work.aw[kAnalogs - 1][z]);
                }
                cf[4] = x;
                x = work.am[kAnalogs - 1][z];
                const float bgSigma = std::sqrt(work.bv[z]);
                x /= bgSigma;
                cf[5] = satlin_sse(cfg.min_analog_snr_thresh0, cfg.min_analog_snr_thresh1, x);
                if (cfg.snr_drop_thresh < 0.0f) cf[6] = 1.0f;
                else
                {
                    const float snrEst = work.am[0][z] / bgSigma;
                    const float r0 = det.am[0][z], r1 = det.am[1][z];
                    const float refBgSigma = std::sqrt(det.bv[z]);
                    assertOk &= (r0 >= 0.0f) & (r1 >= 0.0f) & (refBgSigma >= 0.0f);
                    const float refSnr0 = r0 / refBgSigma;
                    float refSnr1 = r1 / refBgSigma;
                    refSnr1 *= cfg.snr_drop_thresh;
                    refSnr1 *= fmin_sse(det.conf[z], 1.0f);
                    assertOk &= (refSnr1 < refSnr0);
                    cf[6] = satlin_sse(refSnr1, std::sqrt(refSnr0 * refSnr1), snrEst);
                }
                cf[7] = 1.0f;
                float cc = 1.0f;
                for (int k = 0; k < 8; ++k) cc *= cf[k];
                cc = fmin_sse(fmax_sse(0.0f, cc), 1.0f);
                cc = (cc >= cfg.success_confidence_thresh) ? cc : 0.0f;
                conf[z] = cc;
                work.conf[z] = cc;
            }
            if (!assertOk)
            {
#pragma omp critical
                { status = HW_ERR_NUMERIC; errMsg = "DME: Bad threshold in SNR Drop confidence factor"; }
            }
            ModelUpdate(c, det, work);
            ModelToLane(det, models[l]);
            if (diag)
            {
                FZ
                {
                    diag[l].iter_count[z] = mIter[z];
                    diag[l].converged[z] = mConverged[z] ? 1 : 0;
                    diag[l].log_like[z] = mLogLike[z];
                    diag[l].status[z] = zStatus[z];
                    diag[l].confidence[z] = conf[z];
                }
                diag[l].lane_iterations = laneIters;
            }
        }
    }
    if (status != HW_OK) g_err = errMsg;
    return status;
}

// ---------------------------------------------------------------------------
// Single-ZMW EM fit for the learned initializer (no counterpart in the
// reference): the reference's EM steps from the plain start, from a proposal
// or from the one of the two with the higher log-likelihood, run for maxIter
// iterations per ZMW without the lane-wide stop and without the final
// confidence blend.  Layouts per lane: proposal/target/params [15][64]
// (fractions, means, variances of the baseline and four analog modes),
// iters [5][64] (first converged iteration or -1, first iteration within tol
// of the target or -1, fell back to the plain start, status bits, iterations
// until one update first changes the parameters by at most tol), loglike
// [3][64] (plain start, chosen start, last E-step).

// Largest relative distance of one ZMW's parameters from the target, with
// floors 0.01 (fractions), 1 DN (means) and 1 DN^2 (variances).
static float EmDistance(const float rho[5][kLane], const float mu[5][kLane], const float var[5][kLane],
                        const float* t, int z)
{
    float dmax = 0.0f;
    for (int k = 0; k < 5; ++k)
    {
        const float tr = t[k * kLane + z], tm = t[(5 + k) * kLane + z], tv = t[(10 + k) * kLane + z];
        dmax = std::max(dmax, std::abs(rho[k][z] - tr) / std::max(std::abs(tr), 0.01f));
        dmax = std::max(dmax, std::abs(mu[k][z] - tm) / std::max(std::abs(tm), 1.0f));
        dmax = std::max(dmax, std::abs(var[k][z] - tv) / std::max(std::abs(tv), 1.0f));
    }
    return dmax;
}

int OraclePool::EmFit(const hw_lane_histogram* hh, const hw_baseliner_stats* stats, hw_frame_interval hfi,
                      hw_frame_interval pfi, const hw_lane_model* models, int mode, const float* proposal,
                      const float* target, float tol, uint32_t maxIter, float* params, int32_t* iters,
                      float* loglike, float* atStop)
{
    if (mode < 0 || mode > 2 || (mode != 0 && !proposal))
    { g_err = "EmFit: bad start mode or missing proposal"; return HW_ERR_INVALID_ARG; }
    const DmeCtx c{&cfg, &d};
    const int nModes = kAnalogs + 1;
    const int nB = kBins;
#pragma omp parallel
    {
        std::vector<float> tau((size_t)nModes * (nB + 1) * kLane);
        std::vector<float> bprob((size_t)(nB + 1) * kLane), binProb((size_t)nB * kLane), nj((size_t)nB * kLane);
#pragma omp for schedule(dynamic, 1)
        for (int64_t l = 0; l < (int64_t)lanes; ++l)
        {
            auto emPtr = std::make_unique<LaneEm>(c, hh[l], tau.data(), bprob.data(), binProb.data(), nj.data());
            LaneEm& em = *emPtr;
            Model det;
            DmePrelude(l, hh, stats, hfi, pfi, models, det, &em);
            UHist hist{&hh[l]};
            float* P = params + (size_t)l * 15 * kLane;
            int32_t* I = iters + (size_t)l * 5 * kLane;
            float* L = loglike + (size_t)l * 3 * kLane;
            const float* T = target ? target + (size_t)l * 15 * kLane : nullptr;

            float llPlain[kLane], ll[kLane];
            int32_t fellBack[kLane], zStatus[kLane], tolIter[kLane], mIter[kLane], stepIter[kLane];
            float llStart[kLane];
            if (mode != 0)
                em.ChooseStart(proposal + (size_t)l * 15 * kLane, mode == 2, fellBack, llPlain, llStart);
            else
            {
                em.EStep(llPlain);
                FZ { fellBack[z] = 0; llStart[z] = llPlain[z]; }
            }
            float logLike[kLane], mLogLike[kLane], last[kLane];
            bool mConverged[kLane];
            FZ
            {
                zStatus[z] = (hist.Total(z) < 160u) ? 2 : 0;
                tolIter[z] = -1; stepIter[z] = -1; mIter[z] = 0; mConverged[z] = false;
                logLike[z] = std::numeric_limits<float>::lowest();
                mLogLike[z] = -kInf;
                last[z] = llStart[z];
            }
            for (uint32_t it = 0; it < maxIter; ++it)
            {
                if (T)
                    FZ if (tolIter[z] < 0 && EmDistance(em.rho, em.mu, em.var, T, z) <= tol) tolIter[z] = (int32_t)it;
                em.EStep(ll);
                FZ
                {
                    const float prev = logLike[z];
                    logLike[z] = ll[z];
                    const float delta = ll[z] - prev;
                    const float convTol = 1e-4f * fmax_sse(ll[z], -ll[z]);
                    bool cv = (delta >= 0) & (delta < convTol);
                    cv &= (ll[z] >= mLogLike[z]);
                    mIter[z] = (cv & !mConverged[z]) ? (int32_t)it : mIter[z];
                    if (atStop && cv && !mConverged[z])
                    {
                        float* S = atStop + (size_t)l * 15 * kLane;
                        for (int k = 0; k < 5; ++k)
                        {
                            S[k * kLane + z] = em.rho[k][z];
                            S[(5 + k) * kLane + z] = em.mu[k][z];
                            S[(10 + k) * kLane + z] = em.var[k][z];
                        }
                    }
                    mLogLike[z] = cv ? ll[z] : mLogLike[z];
                    mConverged[z] |= cv;
                    last[z] = ll[z];
                }
                float rhoB[5][kLane], muB[5][kLane], varB[5][kLane];
                std::memcpy(rhoB, em.rho, sizeof(rhoB));
                std::memcpy(muB, em.mu, sizeof(muB));
                std::memcpy(varB, em.var, sizeof(varB));
                em.MStep(zStatus);
                FZ
                {
                    float dmax = 0.0f;
                    for (int k = 0; k < 5; ++k)
                    {
                        dmax = std::max(dmax, std::abs(em.rho[k][z] - rhoB[k][z]) / std::max(std::abs(em.rho[k][z]), 0.01f));
                        dmax = std::max(dmax, std::abs(em.mu[k][z] - muB[k][z]) / std::max(std::abs(em.mu[k][z]), 1.0f));
                        dmax = std::max(dmax, std::abs(em.var[k][z] - varB[k][z]) / std::max(std::abs(em.var[k][z]), 1.0f));
                    }
                    if (stepIter[z] < 0 && dmax <= tol) stepIter[z] = (int32_t)it + 1;
                }
            }
            if (T)
                FZ if (tolIter[z] < 0 && EmDistance(em.rho, em.mu, em.var, T, z) <= tol) tolIter[z] = (int32_t)maxIter;
            if (atStop)
                FZ if (!mConverged[z])
                    for (int k = 0; k < 15; ++k) atStop[(size_t)l * 15 * kLane + k * kLane + z] = std::nanf("");
            FZ
            {
                for (int k = 0; k < 5; ++k)
                {
                    P[k * kLane + z] = em.rho[k][z];
                    P[(5 + k) * kLane + z] = em.mu[k][z];
                    P[(10 + k) * kLane + z] = em.var[k][z];
                }
                I[0 * kLane + z] = mConverged[z] ? mIter[z] : -1;
                I[1 * kLane + z] = tolIter[z];
                I[2 * kLane + z] = fellBack[z];
                I[3 * kLane + z] = zStatus[z];
                I[4 * kLane + z] = stepIter[z];
                L[0 * kLane + z] = llPlain[z];
                L[1 * kLane + z] = llStart[z];
                L[2 * kLane + z] = last[z];
            }
        }
    }
    return HW_OK;
}

// ---------------------------------------------------------------------------
// Frame labeler: TA/FrameLabelerHost.cpp:54-612, TA/SubframeScorer.h,
// TA/RoiHost.h

namespace {

// BlockStateSubframeScorer (SubframeScorer.h:152-318), one ZMW.
struct Scorer
{
    float bgMean, bInvVar, bgFixed, x0;
    float ffMean[4], pInvVar[4], ffFixed[4], logPMean[4], x1[4];
    float fbMean, fbVar, fbNormTerm, fbScale;

    void Setup(const hwp::Derived& d, const hw_lane_model& m, int z)
    {
        constexpr float log2pi_f = 1.8378770664f;
        const float nhalf = -0.5f;
        const float halfVal = 0.5f, oneSixth = 1.0f / 6.0f;
        const float bMean = f16_bits_to_f32(m.baseline.means[z]);
        const float bVar = f16_bits_to_f32(m.baseline.vars[z]);
        const float bSigma = std::sqrt(bVar);
        x0 = bMean + bSigma * d.sqrtHalfPi;
        bInvVar = 1.0f / bVar;
        for (int a = 0; a < kAnalogs; ++a)
        {
            const float aMean = f16_bits_to_f32(m.analogs[a].means[z]);
            logPMean[a] = hw_logf(aMean - bMean);
            const float aVar = f16_bits_to_f32(m.analogs[a].vars[z]);
            const float aSigma = std::sqrt(aVar);
            x1[a] = aMean - aSigma * d.sqrtHalfPi;
            pInvVar[a] = 1.0f / aVar;
        }
        {
            const float aMean = f16_bits_to_f32(m.analogs[3].means[z]);
            const float aVar = f16_bits_to_f32(m.analogs[3].vars[z]);
            float eMean = halfVal * (bMean + aMean);
            float eVar = oneSixth * (aMean - bMean);
            eVar += bVar + aVar;
            eVar *= halfVal;
            fbMean = eMean;
            fbVar = eVar;
            // NormalLog::operator() (SubframeScorer.h:117-123); its two
            // data-independent terms are the same on every call.
            fbNormTerm = -0.5f * (log2pi_f + hw_logf(fbVar));
            fbScale = 0.5f / fbVar;
        }
        const float normConst = log2pi_f / 2.0f;
        bgFixed = nhalf * hw_logf(bVar) - normConst;
        bgMean = bMean;
        for (int i = 0; i < kAnalogs; ++i)
        {
            const float aVar = f16_bits_to_f32(m.analogs[i].vars[z]);
            ffFixed[i] = nhalf * hw_logf(aVar) - normConst;
            ffMean[i] = f16_bits_to_f32(m.analogs[i].means[z]);
        }
    }

    // SubframeScore, SubframeScorer.h:264-295
    float Subframe(int a, float val) const
    {
        const float nhalf = -0.5f;
        const bool lowExtrema = val < x0;
        const float cap = lowExtrema ? x0 : x1[a];
        float fixedTerm = lowExtrema ? bInvVar : pInvVar[a];
        fixedTerm = nhalf * fixedTerm;
        const bool extrema = lowExtrema | (val > x1[a]);
        const float dv = val - cap;
        float s = (extrema ? fixedTerm * (dv * dv) : 0.0f) - logPMean[a];
        if (a == kAnalogs - 1)
        {
            const float dm = val - fbMean;
            const float fb = fbNormTerm - (dm * dm) * fbScale;
            s = (x0 <= x1[a]) ? s : fb;
        }
        return s;
    }

    // StateScores, SubframeScorer.h:185-228
    void Scores(float data, float* out) const
    {
        const float nhalf = -0.5f;
        {
            const float y = data - bgMean;
            out[0] = nhalf * y * bInvVar * y + bgFixed;
        }
        float full[4];
        for (int i = 0; i < 4; ++i)
        {
            const float y = data - ffMean[i];
            full[i] = nhalf * y * pInvVar[i] * y + ffFixed[i];
            out[1 + i] = full[i];
        }
        for (int i = 0; i < 4; ++i)
        {
            float score = Subframe(i, data);
            score = (data > ffMean[i]) ? fmin_sse(fmin_sse(score, full[i] - 1.0f), 0.0f) : score;
            out[5 + i] = score;
            out[9 + i] = score;
        }
    }
};

}   // namespace

// margin (optional, [lanes][F][64]): the best path's decision margin of each
// label.  Label f < F - 1 is the arg-max source that the Viterbi step of frame
// f + 1 recorded for the path's state there; its margin is that step's gap
// between the winning candidate and the best other one of the state's row
// (0 on a tie, +inf with a single finite candidate).  The last label is the
// anchor state; its margin is the gap between the largest back-propagated
// end-state probability and the next largest.
int OraclePool::Label(const int16_t* traces, const hw_lane_model* models, int16_t* labels,
                      int16_t* latOut, float* score, float* margin)
{
    const int L = hwp::kLatentFrames;
    const int LB = hwp::kViterbiStitchLookback;
    const int nRoi = (int)F + LB + hwp::kRoiStitchFrames;   // roi workspace frames
    const hwp::SparseRows sp = hwp::TransitionPattern();
    const bool roiNoop = (cfg.roi_filter_type == HW_ROI_NOOP);
    if (roiNoop) { g_err = "RoiFilterNoOp is not built"; return HW_ERR_UNSUPPORTED; }

#pragma omp parallel
    {
        std::vector<uint16_t> tb((size_t)(F + LB) * kStates);   // traceback per frame per state
        std::vector<float> gap(margin ? (size_t)(F + LB) * kStates : 0);   // decision gap per frame per state
        std::vector<uint8_t> roi(nRoi);
        std::vector<float> tr((size_t)(F + L));
#pragma omp for schedule(dynamic, 1)
        for (int64_t l = 0; l < (int64_t)lanes; ++l)
        {
            const int16_t* chunk = traces + (size_t)l * F * kLane;
            int16_t* pl = &prevLat[(size_t)l * L * kLane];
            const hw_lane_model& oldM = latModel[l];
            const hw_lane_model& newM = models[l];
            for (int z = 0; z < kLane; ++z)
            {
                // ComputeRoi (FrameLabelerHost.cpp:267-309, RoiHost.h:110-249)
                const float inv1 = 1 / std::sqrt(f16_bits_to_f32(oldM.baseline.vars[z]));
                const float inv2 = 1 / std::sqrt(f16_bits_to_f32(newM.baseline.vars[z]));
                float prev[3];
                prev[0] = (float)latTrc[(size_t)l * kLane + z] * inv1;
                prev[1] = (float)pl[0 * kLane + z] * inv1;
                prev[2] = (float)pl[1 * kLane + z] * inv1;
                uint16_t prevRoi = (uint16_t)latRoi[(size_t)l * kLane + z];
                int ri = 0;
                auto process = [&](float sn) {
                    float mval = prev[1];
                    mval = fmax_sse(mval, (prev[0] + prev[1]) / d.sqrt2);
                    mval = fmax_sse(mval, (prev[0] + prev[1] + prev[2]) / d.sqrt3);
                    mval = fmax_sse(mval, (prev[0] + prev[1] + prev[2] + sn) / 2.0f);
                    const float thresh = (prevRoi & 1u) ? cfg.roi_lower_threshold : cfg.roi_upper_threshold;
                    const uint16_t v1 = (mval >= thresh) ? 1u : 0u;
                    const uint16_t v2 = (mval >= cfg.roi_lower_threshold) ? 2u : 0u;
                    const uint16_t v = v1 | v2;
                    roi[ri++] = (uint8_t)v;
                    prevRoi = v;
                    prev[0] = prev[1]; prev[1] = prev[2]; prev[2] = sn;
                };
                for (int i = hwp::kRoiLookForward; i < L; ++i) process((float)pl[(size_t)i * kLane + z] * inv1);
                for (int i = 0; i < (int)F; ++i) process((float)chunk[(size_t)i * kLane + z] * inv2);
                {
                    uint16_t pr = 0;
                    for (int i = nRoi - 1; i >= 0; --i)
                    {
                        const bool b = (roi[i] & 1u) | ((roi[i] & 2u) && pr != 0);
                        pr = b ? 1u : 0u;
                        roi[i] = b ? 1u : 0u;
                    }
                }

                // LabelBlock (FrameLabelerHost.cpp:314-448)
                float ll[kStates], la[kStates];
                const int bc = latLabel[(size_t)l * kLane + z];
                for (int i = 0; i < kStates; ++i) ll[i] = (bc == i) ? 0.0f : -kInf;
                for (int f = 0; f < L; ++f) tr[f] = (float)pl[(size_t)f * kLane + z];
                for (int f = 0; f < (int)F; ++f) tr[L + f] = (float)chunk[(size_t)f * kLane + z];

                Scorer sc;
                float anchorLL[kStates];
                auto recursion = [&](int lf, float data) {
                    float sco[kStates];
                    sc.Scores(data, sco);
                    const bool isRoi = roi[lf] != 0;
                    for (int r = 0; r < kStates; ++r)
                    {
                        const float score = sco[r];
                        int idx = sp.first[r];
                        float mv = score + d.trans[r][idx] + ll[idx];
                        float sv = -kInf;     // best of the other candidates
                        for (int p = sp.segBegin[r]; p < sp.segEnd[r]; ++p)
                        {
                            const float v = score + d.trans[r][p] + ll[p];
                            const bool cnd = v >= mv;
                            sv = cnd ? mv : ((v > sv) ? v : sv);
                            mv = cnd ? v : mv;
                            idx = cnd ? p : idx;
                        }
                        const float penalty = (r == 0 || isRoi) ? 0.0f : kInf;
                        la[r] = mv - penalty;
                        tb[(size_t)lf * kStates + r] = (uint16_t)idx;
                        if (margin) gap[(size_t)lf * kStates + r] = mv - sv;
                    }
                    for (int r = 0; r < kStates; ++r) ll[r] = la[r];
                };
                sc.Setup(d, oldM, z);
                for (int f = 0; f < L; ++f) recursion(f, tr[f]);
                sc.Setup(d, newM, z);
                const int anchor = (int)F - L;
                for (int f = 0; f < anchor; ++f) recursion(f + L, tr[L + f]);
                for (int i = 0; i < kStates; ++i) anchorLL[i] = ll[i];
                for (int f = anchor; f < anchor + LB; ++f) recursion(f + L, tr[L + f]);

                // Normalize (FrameLabelerHost.cpp:186-205)
                float prob[kStates];
                {
                    float mx = ll[0];
                    for (int i = 1; i < kStates; ++i) mx = fmax_sse(ll[i], mx);
                    float sum = 0.0f;
                    for (int i = 0; i < kStates; ++i) { prob[i] = hw_expf(ll[i] - mx); sum += prob[i]; }
                    const float inv = 1 / sum;
                    for (int i = 0; i < kStates; ++i) prob[i] *= inv;
                }
                for (int i = (int)F + LB - 1; i > (int)F - 1; --i)
                {
                    float np[kStates];
                    for (int s = 0; s < kStates; ++s) np[s] = 0.0f;
                    for (int from = 0; from < kStates; ++from)
                        np[tb[(size_t)i * kStates + from]] += prob[from];
                    for (int s = 0; s < kStates; ++s) prob[s] = np[s];
                }
                float maxP = prob[0];
                int anchorState = 0;
                for (int i = 1; i < kStates; ++i)
                {
                    const bool cnd = maxP > prob[i];
                    maxP = cnd ? maxP : prob[i];
                    anchorState = cnd ? anchorState : i;
                }
                int ts = anchorState;
                int16_t* out = labels + (size_t)l * F * kLane;
                float* mg = margin ? margin + (size_t)l * F * kLane : nullptr;
                if (mg)
                {
                    float second = -kInf;
                    for (int i = 0; i < kStates; ++i)
                        if (i != anchorState) second = (prob[i] > second) ? prob[i] : second;
                    mg[(size_t)(F - 1) * kLane + z] = maxP - second;
                }
                for (int f = (int)F - 1; f >= 0; --f)
                {
                    out[(size_t)f * kLane + z] = (int16_t)ts;
                    if (mg && f < (int)F - 1)
                        mg[(size_t)f * kLane + z] = gap[(size_t)(f + 1) * kStates + out[(size_t)(f + 1) * kLane + z]];
                    ts = tb[(size_t)f * kStates + ts];
                }
                latRoi[(size_t)l * kLane + z] = roi[F - 1];
                latLabel[(size_t)l * kLane + z] = (int16_t)anchorState;
                latTrc[(size_t)l * kLane + z] = chunk[(size_t)(anchor - 1) * kLane + z];
                if (score) score[(size_t)l * kLane + z] = anchorLL[anchorState];
            }
            // LatentTrace of the returned batch = traces the first 24 labels
            // belong to; then the latent buffer advances to this chunk's tail.
            if (latOut) std::memcpy(latOut + (size_t)l * L * kLane, pl, sizeof(int16_t) * L * kLane);
            std::memcpy(pl, chunk + (size_t)(F - L) * kLane, sizeof(int16_t) * L * kLane);
            latModel[l] = newM;
        }
    }
    return HW_OK;
}

// ---------------------------------------------------------------------------
// Pulse accumulator: TA/HostPulseAccumulator.{h,cpp}, DT/Pulse.h,
// DT/BatchVectors.h:105-119

namespace {
inline uint16_t ToFixed(float v) { return static_cast<uint16_t>(v / .1f + 0.5f); }
}

int OraclePool::Pulses(const int16_t* labels, const int16_t* latTrace, const int16_t* trace, int32_t firstFrame,
                       const hw_lane_model* models, hw_pulse* pulses, uint32_t* lens, uint32_t* ovf,
                       hw_stat_accum_state* blstats)
{
    const int L = hwp::kLatentFrames;
    const uint32_t cap = cfg.max_calls_per_zmw;
    const float maxSignal = 65535 * .1f;
    const float minSignal = 0.0f;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t l = 0; l < (int64_t)lanes; ++l)
    {
        Segment& s = seg[l];
        StatAcc bs;
        bs.Reset();
        uint32_t* ln = lens + (size_t)l * kLane;
        uint32_t* ov = ovf + (size_t)l * kLane;
        hw_pulse* pz = pulses + (size_t)l * kLane * cap;
        FZ { ln[z] = 0; ov[z] = 0; }
        float minMean[kLane];
        FZ minMean[z] = f16_bits_to_f32(models[l].analogs[kAnalogs - 1].means[z]);
        for (uint32_t rel = 0; rel < F; ++rel)
        {
            const uint32_t absF = rel + (uint32_t)firstFrame;
            const int16_t* lab = labels + ((size_t)l * F + rel) * kLane;
            const int16_t* sig = (rel < (uint32_t)L) ? latTrace + ((size_t)l * L + rel) * kLane
                                                     : trace + ((size_t)l * F + (rel - L)) * kLane;
            FZ
            {
                const int16_t label = lab[z];
                const int16_t signal = sig[z];
                const bool isUp = (label > kAnalogs) & (label <= 2 * kAnalogs);
                const bool boundary = isUp | ((label == 0) & (s.label[z] != 0));
                const bool pulseM = s.label[z] != 0;
                if (boundary & pulseM)
                {
                    // LabelsSegment::ToPulse (HostPulseAccumulator.h:106-138)
                    const int width = (int)(absF - s.start[z]);
                    const float rawMean = float(s.total[z] + s.last[z] + s.first[z]) / width;
                    const float rawMid = float(s.total[z]) / (width - 2);
                    const bool keep = (width >= d.widthThresh) || (rawMean * width >= d.ampThresh * minMean[z]);
                    hw_pulse p;
                    std::memset(&p, 0, sizeof(p));
                    p.start = s.start[z];
                    p.width = (uint16_t)width;
                    p.mean_signal = ToFixed(std::min(maxSignal, std::max(minSignal, rawMean)));
                    p.mid_signal = ToFixed(width < 3 ? 0.0f : std::min(maxSignal, std::max(minSignal, rawMid)));
                    p.max_signal = ToFixed(std::min(maxSignal, std::max(minSignal, static_cast<float>(s.mx[z]))));
                    p.signal_m2 = s.m2[z];
                    int lb = s.label[z];
                    if (lb > 2 * kAnalogs) lb -= 2 * kAnalogs;
                    if ((lb > kAnalogs) & (lb <= 2 * kAnalogs)) lb -= kAnalogs;
                    p.label = d.analogMap[lb - 1];
                    p.is_reject = keep ? 0 : 1;
                    if (ln[z] < cap) pz[(size_t)z * cap + ln[z]++] = p;
                    else ov[z]++;
                }
                // ResetSegment / AddSignal (HostPulseAccumulator.h:140-161)
                if (boundary)
                {
                    s.start[z] = absF; s.end[z] = 0; s.first[z] = signal; s.last[z] = 0;
                    s.mx[z] = signal; s.total[z] = 0.0f; s.m2[z] = 0.0f; s.label[z] = label;
                }
                else
                {
                    s.total[z] = s.total[z] + s.last[z];
                    s.m2[z] = s.m2[z] + float(s.last[z]) * s.last[z];
                    s.last[z] = signal;
                    s.mx[z] = std::max(s.mx[z], signal);
                }
                const bool isBl = (!pulseM) & (!boundary);
                bs.AddMasked(z, (float)signal, isBl);
            }
        }
        bs.Store(blstats[l]);
    }
    return HW_OK;
}

// ---------------------------------------------------------------------------
// C API for ctypes (tests and bench.py only)

extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

int or_config_default(hw_config* c) { hwp::DefaultConfig(c); return HW_OK; }

int or_transition_matrix(const hw_config* c, float* out)
{
    float t[kStates][kStates];
    hwp::TransitionMatrix(*c, t);
    std::memcpy(out, t, sizeof(t));
    return HW_OK;
}

void* or_pool_create(const hw_config* cfg, uint32_t poolId, uint32_t lanes, uint32_t F)
{
    auto p = std::make_unique<OraclePool>();
    if (!p->Init(*cfg, poolId, lanes, F)) return nullptr;
    return p.release();
}

void or_pool_destroy(void* p) { delete static_cast<OraclePool*>(p); }

int or_set_threads(int n) { if (n > 0) omp_set_num_threads(n); return omp_get_max_threads(); }

uint32_t or_baseliner_startup_latency(void* p) { return static_cast<OraclePool*>(p)->d.baselinerStartupLatency; }

int or_baseline(void* p, const int16_t* trace, int32_t firstFrame, int16_t* out, hw_baseliner_stats* stats)
{ return static_cast<OraclePool*>(p)->Baseline(trace, firstFrame, out, stats); }

int or_agg_add(void* p, const hw_baseliner_stats* s, hw_frame_interval fi)
{ static_cast<OraclePool*>(p)->AggAdd(s, fi); return HW_OK; }

int or_agg_get(void* p, hw_baseliner_stats* out, hw_frame_interval* fi)
{ static_cast<OraclePool*>(p)->AggGet(out, fi); return HW_OK; }

int or_agg_reset(void* p) { static_cast<OraclePool*>(p)->AggReset(); return HW_OK; }

int or_hist_reset_from_stats(void* p, const hw_baseliner_stats* s)
{ return static_cast<OraclePool*>(p)->HistResetStats(s); }

int or_hist_reset_from_bounds(void* p, const hw_lane_hist_bounds* b)
{ return static_cast<OraclePool*>(p)->HistResetBounds(b); }

int or_hist_add(void* p, const int16_t* tr, uint32_t frames, hw_frame_interval fi, const hw_lane_model* m)
{ return static_cast<OraclePool*>(p)->HistAdd(tr, frames, fi, m); }

int or_hist_get(void* p, hw_lane_histogram* out, hw_frame_interval* fi)
{ static_cast<OraclePool*>(p)->HistGet(out, fi); return HW_OK; }

int or_dme_init_models(void* p, const hw_baseliner_stats* s, hw_lane_model* out)
{ static_cast<OraclePool*>(p)->InitModels(s, out); return HW_OK; }

int or_dme_estimate(void* p, const hw_lane_histogram* h, const hw_baseliner_stats* s, hw_frame_interval hfi,
                    hw_frame_interval mfi, hw_lane_model* m, hw_dme_diag* diag)
{ return static_cast<OraclePool*>(p)->Estimate(h, s, hfi, mfi, m, diag); }

int or_label(void* p, const int16_t* tr, const hw_lane_model* m, int16_t* labels, int16_t* latOut, float* score,
             float* margin)
{ return static_cast<OraclePool*>(p)->Label(tr, m, labels, latOut, score, margin); }

int or_pulses(void* p, const int16_t* labels, const int16_t* lat, const int16_t* tr, int32_t firstFrame,
              const hw_lane_model* m, hw_pulse* pulses, uint32_t* lens, uint32_t* ovf, hw_stat_accum_state* bs)
{ return static_cast<OraclePool*>(p)->Pulses(labels, lat, tr, firstFrame, m, pulses, lens, ovf, bs); }

int or_dme_estimate_proposal(void* p, const hw_lane_histogram* h, const hw_baseliner_stats* s, hw_frame_interval hfi,
                             hw_frame_interval mfi, hw_lane_model* m, hw_dme_diag* diag, const float* proposal)
{
    return static_cast<OraclePool*>(p)->Estimate(h, s, hfi, mfi, m, diag, proposal);
}

int or_em_fit(void* p, const hw_lane_histogram* h, const hw_baseliner_stats* s, hw_frame_interval hfi,
              hw_frame_interval mfi, const hw_lane_model* m, int mode, const float* proposal, const float* target,
              float tol, uint32_t maxIter, float* params, int32_t* iters, float* loglike, float* atStop)
{
    return static_cast<OraclePool*>(p)->EmFit(h, s, hfi, mfi, m, mode, proposal, target, tol, maxIter, params,
                                              iters, loglike, atStop);
}

// The fixed detection model of FixedModelBatchAnalyzer, one lane.
int or_static_model(const hw_config* c, hw_lane_model* out)
{
    hwp::StaticModel(*c, out);
    return HW_OK;
}

// One BlockFilterStage (TraceFilters.cpp:11-57 on a WindowBuffer that starts
// with `width` zeros) with stride 1 over `chunks` consecutive blocks of F
// frames of one lane: in/out[chunks][F][64].  Pins the window semantics
// against the reference's extrema-filter sawtooth test.
int or_extremum_stage(int width, int isMax, const int16_t* in, int F, int chunks, int16_t* out)
{
    if (width < 1 || F < 1 || chunks < 0) { g_err = "or_extremum_stage: bad size"; return HW_ERR_INVALID_ARG; }
    Stage st;
    st.spec = hwp::StageSpec{width, 1, 1, isMax != 0};
    st.wb.Init(width);
    std::vector<int16_t> block((size_t)F * kLane);
    for (int c = 0; c < chunks; ++c)
    {
        std::memcpy(block.data(), in + (size_t)c * F * kLane, sizeof(int16_t) * block.size());
        st.Run(block.data(), F);
        std::memcpy(out + (size_t)c * F * kLane, block.data(), sizeof(int16_t) * block.size());
    }
    return HW_OK;
}

float or_expf(float x) { return hw_expf(x); }
float or_logf(float x) { return hw_logf(x); }
uint16_t or_f32_to_f16(float x) { return f32_to_f16_bits(x); }
int16_t or_to_i16(float x) { return to_i16_wrap(x); }

// The workloads' synthetic trace generator (hw_b200/csrc/gen.cu) on the host:
// the same counter-based hash per (seed, ZMW, frame, slot), polar normals and
// float arithmetic, so a chunk is byte-identical to the device generator's.
// It lets the CPU baseline draw its traces without the CUDA library.  The
// workload defaults restate hw_gen_params_default; a test checks both.
namespace {
inline uint64_t GenMix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}
inline uint64_t GenDraw(uint64_t key, uint64_t ctr) { return GenMix64(key ^ GenMix64(ctr)); }
inline float GenU24(uint64_t r, int half)
{
    const uint32_t v = half ? (uint32_t)(r >> 40) : (uint32_t)((r >> 8) & 0xFFFFFFu);
    return (float)v * 5.9604644775390625e-08f;
}
inline float GenNormal(uint64_t key, uint64_t ctrBase)
{
    for (int a = 0; a < 8; ++a)
    {
        const uint64_t r = GenDraw(key, ctrBase + a);
        const float u = 2.0f * GenU24(r, 0) - 1.0f, v = 2.0f * GenU24(r, 1) - 1.0f;
        const float s = u * u + v * v;
        if (s > 0.0f && s < 1.0f) return u * std::sqrt(-2.0f * hw_logf(s) / s);
    }
    return 0.0f;
}

struct OracleGen
{
    hw_gen_params p;
    uint32_t lanes;
    uint64_t zmwOffset;
    std::vector<uint8_t> inPulse;
    std::vector<float> amp, walk;
};
}   // namespace

extern "C" {

int or_gen_params_default(int workload, hw_gen_params* p)
{
    if (!p) return HW_ERR_INVALID_ARG;
    std::memset(p, 0, sizeof(*p));
    p->seed = 0x5eed0000ull + (uint64_t)workload;
    p->baseline_mean = 200.0f;
    p->baseline_sigma = 8.0f;
    const float amps[4] = {80.0f, 50.0f, 32.0f, 20.0f};
    for (int a = 0; a < 4; ++a) p->amplitudes[a] = amps[a];
    p->amp_cv = 0.1f;
    p->pulse_width_mean = 8.0f;
    p->ipd_mean = 14.0f;
    p->shot_coeff = 0.5f;
    p->step_frame = -1;
    switch (workload)
    {
    case 0: break;
    case 1: p->gain_sigma = 0.2f; p->empty_fraction = 0.15f; p->walk_sigma = 0.05f; break;
    case 2: p->amp_scale_sigma = 0.3f; p->rate_min = 0.02f; p->rate_max = 0.12f; p->pulse_width_mean = 4.0f; break;
    case 4:
        p->gain_sigma = 0.2f; p->empty_fraction = 0.15f; p->walk_sigma = 0.05f;
        p->decay_fraction = 0.2f; p->decay_frames = 128 * 512;
        p->step_frame = 64 * 512; p->step_dn = 15.0f; p->step_fraction = 0.01f;
        break;
    default: return HW_ERR_INVALID_ARG;
    }
    return HW_OK;
}

void* or_gen_create(const hw_gen_params* p, uint32_t lanes, uint64_t zmwOffset)
{
    if (!p || lanes == 0) return nullptr;
    auto g = new OracleGen{*p, lanes, zmwOffset, {}, {}, {}};
    const size_t n = (size_t)lanes * kLane;
    g->inPulse.assign(n, 0);
    g->amp.assign(n, 0.0f);
    g->walk.assign(n, 0.0f);
    return g;
}

void or_gen_destroy(void* g) { delete static_cast<OracleGen*>(g); }

// Frames [firstFrame, firstFrame + frames) of every lane into out[lanes][frames][64].
int or_gen_next(void* gp, int16_t* out, int64_t firstFrame, uint32_t frames)
{
    OracleGen& G = *static_cast<OracleGen*>(gp);
    const hw_gen_params& P = G.p;
    const int64_t n = (int64_t)G.lanes * kLane;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < n; ++g)
    {
        const int64_t l = g / kLane, z = g % kLane;
        const uint64_t zmw = G.zmwOffset + (uint64_t)g;
        const uint64_t key = GenMix64(P.seed ^ GenMix64(zmw * 0x2545F4914F6CDD1Dull + 1));
        const float gain = (P.gain_sigma > 0.0f) ? hw_expf(P.gain_sigma * GenNormal(key, 0)) : 1.0f;
        const float ampScale = (P.amp_scale_sigma > 0.0f) ? hw_expf(P.amp_scale_sigma * GenNormal(key, 8)) : 1.0f;
        const uint64_t rz = GenDraw(key, 16);
        const bool empty = GenU24(rz, 0) < P.empty_fraction;
        const bool stepped = GenU24(rz, 1) < P.step_fraction;
        float startHazard = 1.0f / P.ipd_mean;
        if (P.rate_max > 0.0f)
        {
            const float rate = P.rate_min + (P.rate_max - P.rate_min) * GenU24(GenDraw(key, 17), 0);
            const float gap = std::fmax(1.0f / rate - P.pulse_width_mean, 1.0f);
            startHazard = 1.0f / gap;
        }
        const float endHazard = 1.0f / P.pulse_width_mean;
        bool inp = G.inPulse[g] != 0;
        float amp = G.amp[g];
        float walk = G.walk[g];
        int16_t* o = out + (size_t)l * frames * kLane + z;
        for (uint32_t t = 0; t < frames; ++t)
        {
            const int64_t f = firstFrame + t;
            const uint64_t base = (uint64_t)(f + 1) * 32;
            const uint64_t r0 = GenDraw(key, base);
            const float u = GenU24(r0, 0);
            if (inp)
            {
                if (u < endHazard) inp = false;
            }
            else if (!empty && u < startHazard)
            {
                inp = true;
                int a = (int)(GenU24(r0, 1) * 4.0f);
                a = a > 3 ? 3 : a;
                float decay = 1.0f;
                if (P.decay_frames > 0)
                    decay = 1.0f - P.decay_fraction * std::fmin((float)f / (float)P.decay_frames, 1.0f);
                const float an = GenNormal(key, base + 1);
                amp = std::fmax(P.amplitudes[a] * gain * ampScale * decay * (1.0f + P.amp_cv * an), 0.0f);
            }
            if (P.walk_sigma > 0.0f) walk += P.walk_sigma * GenNormal(key, base + 9);
            const float sig = inp ? amp : 0.0f;
            float level = P.baseline_mean + walk + sig;
            if (stepped && P.step_frame >= 0 && f >= P.step_frame) level += P.step_dn;
            const float sd = std::sqrt(P.baseline_sigma * P.baseline_sigma + P.shot_coeff * sig);
            const float v = std::rint(level + sd * GenNormal(key, base + 17));
            o[(size_t)t * kLane] = (int16_t)std::fmin(std::fmax(v, -32768.0f), 32767.0f);
        }
        G.inPulse[g] = inp ? 1 : 0;
        G.amp[g] = amp;
        G.walk[g] = walk;
    }
    return HW_OK;
}

}   // extern "C"

// PicketFenceGenerator::GenerateSignal (appModules/SimulatedDataSource.cpp:
// 252-323, config SimulatedDataSource.h:176-212): the reference baseliner
// tests' traces.  Signal `idx` seeds its own std::mt19937 (seedFunc = the
// identity); an inter-pulse run of baseline frames floor(N(level, sigma)) +
// pedestal, then a pulse run of the same plus (a uniformly chosen pulse level
// - the baseline level); every run draws from a fresh normal_distribution,
// so no cached second polar value crosses runs.  Run lengths are fixed or
// ceil(exponential(rate)).  The C++ standard library's engine and
// distributions are the reference's own.
int or_picket_fence(uint32_t numFrames, uint64_t idx, int poisson, uint16_t pulseWidth, uint16_t pulseIpd,
                    float widthRate, float ipdRate, int16_t blLevel, int16_t blSigma, const int16_t* levels,
                    int nLevels, int16_t pedestal, int16_t* out)
{
    if (nLevels < 1 || !out) { g_err = "picket fence: no pulse levels"; return HW_ERR_INVALID_ARG; }
    std::mt19937 gen((std::mt19937::result_type)idx);
    auto baseline = [&](uint16_t frames, std::vector<short>& v) {
        std::normal_distribution<> rng(blLevel, blSigma);
        v.clear();
        for (size_t f = 0; f < frames; ++f) v.push_back((short)(std::floor(rng(gen)) + pedestal));
    };
    auto width = [&]() -> uint16_t {
        if (poisson) { std::exponential_distribution<> rng(widthRate); return (uint16_t)std::ceil(rng(gen)); }
        return pulseWidth;
    };
    auto ipd = [&]() -> uint16_t {
        if (poisson) { std::exponential_distribution<> rng(ipdRate); return (uint16_t)std::ceil(rng(gen)); }
        return pulseIpd;
    };
    size_t frame = 0;
    std::vector<short> run;
    while (frame < numFrames)
    {
        const uint16_t nIpd = (uint16_t)std::min<size_t>(numFrames - frame, ipd());
        baseline(nIpd, run);
        for (short v : run) out[frame++] = v;
        const uint16_t nPw = (uint16_t)std::min<size_t>(numFrames - frame, width());
        std::uniform_int_distribution<> pick(0, nLevels - 1);
        const int level = levels[pick(gen)] - blLevel;
        baseline(nPw, run);
        for (short v : run) out[frame++] = (short)(v + level);
    }
    return HW_OK;
}

// DetectionModelHost(ldm, fi) and ExportTo on [lanes][16][64] float
// parameters (baseline weight, mean, variance; analog weight, mean, variance
// each; confidence), and EvolveConfidence on their confidence row.
static void ParamsToModel(const float* p, Model& m)
{
    FZ
    {
        m.bw[z] = p[0 * kLane + z]; m.bm[z] = p[1 * kLane + z]; m.bv[z] = p[2 * kLane + z];
        for (int a = 0; a < kAnalogs; ++a)
        {
            m.aw[a][z] = p[(3 + 3 * a) * kLane + z];
            m.am[a][z] = p[(4 + 3 * a) * kLane + z];
            m.av[a][z] = p[(5 + 3 * a) * kLane + z];
        }
        m.conf[z] = p[15 * kLane + z];
    }
}

static void ModelToParams(const Model& m, float* p)
{
    FZ
    {
        p[0 * kLane + z] = m.bw[z]; p[1 * kLane + z] = m.bm[z]; p[2 * kLane + z] = m.bv[z];
        for (int a = 0; a < kAnalogs; ++a)
        {
            p[(3 + 3 * a) * kLane + z] = m.aw[a][z];
            p[(4 + 3 * a) * kLane + z] = m.am[a][z];
            p[(5 + 3 * a) * kLane + z] = m.av[a][z];
        }
        p[15 * kLane + z] = m.conf[z];
    }
}

int or_detection_model_import(const hw_lane_model* models, uint32_t lanes, float* params)
{
    for (uint32_t l = 0; l < lanes; ++l)
    {
        Model m;
        ModelFromLane(models[l], hw_frame_interval{0, 1}, m);
        ModelToParams(m, params + (size_t)l * 16 * kLane);
    }
    return HW_OK;
}

int or_detection_model_export(const float* params, uint32_t lanes, hw_lane_model* models)
{
    for (uint32_t l = 0; l < lanes; ++l)
    {
        Model m;
        ParamsToModel(params + (size_t)l * 16 * kLane, m);
        ModelToLane(m, models[l]);
    }
    return HW_OK;
}

int or_detection_model_evolve_confidence(float* params, uint32_t lanes, hw_frame_interval from,
                                         hw_frame_interval to, float halfLife)
{
    if (from.lower >= from.upper || to.lower >= to.upper) { g_err = "empty frame interval"; return HW_ERR_INVALID_ARG; }
    for (uint32_t l = 0; l < lanes; ++l)
    {
        Model m;
        float* p = params + (size_t)l * 16 * kLane;
        ParamsToModel(p, m);
        EvolveConfidence(m, CenterInt(from), CenterInt(to), halfLife);
        ModelToParams(m, p);
    }
    return HW_OK;
}

}   // extern "C"

// ===========================================================================
// HF metrics: TA/HFMetricsFilterHost.cpp:40-121,
// DT/BasecallingMetricsAccumulator.cpp:40-504, DT/TraceAnalysisMetrics.h:48-200,
// CM/StatAccumulator.h:80-252 (offset-aware), CM/AutocorrAccumulator.cpp:42-67.
// Lane-wide all()/any() conditions of the SIMD code are evaluated over the
// 64 ZMWs of the lane, as the LaneArray code does.

namespace {

// StatAccumulator with a live offset (the trace metrics' baseline accumulator).
struct HfStat
{
    float off[kLane], m0[kLane], m1[kLane], m2[kLane];
    void Zero() { FZ { off[z] = 0; m0[z] = 0; m1[z] = 0; m2[z] = 0; } }
    void ResetMoments() { FZ { m0[z] = 0; m1[z] = 0; m2[z] = 0; } }     // Reset(): offset kept
    float Mean(int z) const { return m1[z] / m0[z] + off[z]; }
    float Variance(int z) const
    {
        float var = m1[z] * m1[z] / m0[z];
        var = (m2[z] - var) / (m0[z] - 1.0f);
        var = fmax_sse(var, 0.0f);
        return (m0[z] > 1.0f) ? var : kNaN;
    }
    // Offset(value), :234-246
    void SetOffset(const float* value)
    {
        bool same = true;
        FZ same &= (value[z] == off[z]);
        if (same) return;
        FZ
        {
            const float m1new = m1[z] + m0[z] * (off[z] - value[z]);
            const float m2new = m2[z] + (m1new * m1new - m1[z] * m1[z]) / m0[z];
            off[z] = value[z];
            m1[z] = m1new;
            m2[z] = (m0[z] == 0.0f) ? 0.0f : m2new;
        }
    }
    // operator+=(StatAccumulator other), :144-166
    void PlusEq(HfStat other)
    {
        bool allEmpty = true;
        FZ allEmpty &= (other.m0[z] == 0.0f);
        if (allEmpty) return;
        bool anyNan = false;
        FZ anyNan |= std::isnan(off[z]);
        if (anyNan)
        {
            FZ if (std::isnan(off[z])) { m0[z] = 0; m1[z] = 0; m2[z] = 0; }
            FZ off[z] = std::isnan(off[z]) ? 0.0f : off[z];
        }
        float offNew[kLane];
        FZ
        {
            const float w = other.m0[z] / (m0[z] + other.m0[z]);
            const float o = (1.0f - w) * off[z] + w * other.off[z];
            offNew[z] = std::isnan(o) ? off[z] : o;
        }
        other.SetOffset(offNew);
        SetOffset(offNew);
        FZ { m0[z] += other.m0[z]; m1[z] += other.m1[z]; m2[z] += other.m2[z]; }
    }
};

// AutocorrAccumulator::Autocorrelation, AutocorrAccumulator.cpp:42-67
float Autocorrelation(const AutocorrAcc& a, int z)
{
    const float nmk = a.stats.m0[z] - 4.0f;
    const float mu = a.stats.Mean(z) - a.stats.off[z];
    float m1x2 = 2.0f * a.stats.m1[z];
    for (int k = 0; k < 4; ++k) m1x2 -= a.fBuf[k][z] + a.bBuf[k][z];
    float ac = mu * (m1x2 - nmk * mu);
    ac = (a.m2[z] - ac) / ((nmk - 1.0f) * a.stats.Variance(z));
    ac = fmin_sse(fmax_sse(ac, -1.0f), 1.0f);
    return ((nmk < 1.0f) | std::isnan(ac)) ? kNaN : ac;
}

struct HfCart
{
    std::vector<int16_t> left, right;
    std::vector<int8_t> feature, value;
    std::vector<float> thr;
    float hsw[2] = {0, 0};
    float maxHsw = 0;
};

constexpr uint8_t kNoneLabel = 5;     // Pulse::NucleotideLabel::NONE

// One lane's BasecallingMetricsAccumulator.
struct HfLane
{
    uint16_t pulseFrames[kLane], baseFrames[kLane], sandwiches[kLane], halfSandwiches[kLane], stutters[kLane];
    uint8_t activity[kLane];
    float pkMid[4][kLane], bpZvar[4][kLane], pkZvar[4][kLane], pkMax[4][kLane];
    float modelVar[4][kLane], modelMean[4][kLane];
    uint16_t pkMidFrames[4][kLane], pkMidBases[4][kLane], basesBy[4][kLane], pulsesBy[4][kLane];
    // TraceAnalysisMetrics
    uint32_t startFrame[kLane], numFrames[kLane];
    int16_t pixelChecksum[kLane];
    float pdScore[kLane];
    HfStat blStat;
    AutocorrAcc corr;
    hw_pulse prev[kLane], prevprev[kLane];

    void Init()
    {
        FZ { startFrame[z] = 0; numFrames[z] = 0; pixelChecksum[z] = 0; }
        blStat.Zero();
        corr.Reset();
        Reset();
    }
    // BasecallingMetricsAccumulator::Reset, :249-272 + TraceAnalysisMetrics::Reset
    void Reset()
    {
        FZ
        {
            pulseFrames[z] = 0; baseFrames[z] = 0; sandwiches[z] = 0; halfSandwiches[z] = 0; stutters[z] = 0;
            hw_pulse none{};
            none.label = kNoneLabel;
            prev[z] = none;
            prevprev[z] = none;
            activity[z] = 0;
            for (int a = 0; a < 4; ++a)
            {
                pkMid[a][z] = 0; bpZvar[a][z] = 0; pkZvar[a][z] = 0; pkMax[a][z] = 0;
                pkMidFrames[a][z] = 0; pkMidBases[a][z] = 0; basesBy[a][z] = 0; pulsesBy[a][z] = 0;
            }
        }
        blStat.ResetMoments();
        {
            // AutocorrAccumulator::Reset keeps the offset
            float off[kLane];
            FZ off[z] = corr.stats.off[z];
            corr.Reset();
            FZ corr.stats.off[z] = off[z];
        }
        FZ { startFrame[z] = startFrame[z] + numFrames[z]; numFrames[z] = 0; pdScore[z] = 0.0f; }
    }

    static float MidSignal(const hw_pulse& p) { return p.width < 3 ? kNaN : (float)p.mid_signal * 0.1f; }
    static float SignalM2(const hw_pulse& p) { return p.width < 3 ? kNaN : p.signal_m2; }

    // Count, :348-412
    void Count(const hw_pulse* pulses, const uint32_t* lens, uint32_t cap, uint32_t frames)
    {
        FZ numFrames[z] += frames;
        FZ
        {
            const hw_pulse* pp = &prev[z];
            const hw_pulse* ppp = &prevprev[z];
            const hw_pulse* row = pulses + (size_t)z * cap;
            for (uint32_t bi = 0; bi < lens[z]; ++bi)
            {
                const hw_pulse* p = &row[bi];
                const uint8_t lb = p->label;
                pulseFrames[z] = (uint16_t)(pulseFrames[z] + p->width);
                pulsesBy[lb][z]++;
                pkMax[lb][z] = std::max(pkMax[lb][z], (float)p->max_signal * 0.1f);
                if (pp->label != kNoneLabel)
                {
                    if (pp->label == lb) stutters[z]++;
                    const bool abutted = p->start == pp->start + pp->width;
                    if (abutted && pp->label != lb) halfSandwiches[z]++;
                    if (ppp->label != kNoneLabel)
                    {
                        const bool prevAbutted = pp->start == ppp->start + ppp->width;
                        if (prevAbutted && abutted && ppp->label == lb && ppp->label != pp->label) sandwiches[z]++;
                    }
                }
                if (!p->is_reject)
                {
                    baseFrames[z] = (uint16_t)(baseFrames[z] + p->width);
                    basesBy[lb][z]++;
                    if (!std::isnan(MidSignal(*p)))
                    {
                        pkMidBases[lb][z]++;
                        const uint16_t midWidth = (uint16_t)(p->width - 2);
                        pkMidFrames[lb][z] = (uint16_t)(pkMidFrames[lb][z] + midWidth);
                        pkMid[lb][z] += MidSignal(*p) * midWidth;
                        bpZvar[lb][z] += MidSignal(*p) * MidSignal(*p) * midWidth;
                        pkZvar[lb][z] += SignalM2(*p);
                    }
                }
                ppp = pp;
                pp = p;
            }
            prev[z] = *pp;
            prevprev[z] = *ppp;
        }
    }

    // AddModels, :311-322
    void AddModels(const hw_lane_model& m)
    {
        for (int a = 0; a < 4; ++a)
            FZ { modelVar[a][z] = hwm::f16_bits_to_f32(m.analogs[a].vars[z]); modelMean[a][z] = hwm::f16_bits_to_f32(m.analogs[a].means[z]); }
    }

    // AddBatchMetrics, :324-340
    void AddBatchMetrics(const hw_baseliner_stats& bs, const float* viterbi, const hw_stat_accum_state& pd)
    {
        AutocorrAcc sub;
        sub.Load(bs.full_autocorr);
        corr.Merge(sub);
        FZ pdScore[z] += viterbi[z];
        HfStat p;
        FZ { p.off[z] = pd.offset[z]; p.m0[z] = pd.moment0[z]; p.m1[z] = pd.moment1[z]; p.m2[z] = pd.moment2[z]; }
        FZ
        {
            const float bgMean = bs.background_stats.moment1[z] / bs.background_stats.moment0[z]
                               + bs.background_stats.offset[z];
            p.off[z] += bgMean;
        }
        blStat.PlusEq(p);
    }

    uint16_t NumBases(int z) const
    {
        uint16_t r = 0;
        for (int a = 0; a < 4; ++a) r = (uint16_t)(r + basesBy[a][z]);
        return r;
    }
    uint16_t NumPulses(int z) const
    {
        uint16_t r = 0;
        for (int a = 0; a < 4; ++a) r = (uint16_t)(r + pulsesBy[a][z]);
        return r;
    }

    // FinalizeMetrics, :414-500
    void Finalize(bool realtime, float frameRate, const HfCart* cart)
    {
        for (int a = 0; a < 4; ++a)
        {
            bool allZero = true, allFewBases = true, allFewFrames = true;
            FZ
            {
                allZero &= ((int16_t)pkMidBases[a][z] == 0);
                allFewBases &= ((float)pkMidBases[a][z] < 2.0f);
                allFewFrames &= ((float)pkMidFrames[a][z] < 2.0f);
            }
            if (allZero)
            {
                FZ { pkMid[a][z] = kNaN; bpZvar[a][z] = kNaN; pkZvar[a][z] = kNaN; }
            }
            else if (allFewBases || allFewFrames)
            {
                FZ { bpZvar[a][z] = kNaN; pkZvar[a][z] = kNaN; }
            }
            else
            {
                FZ
                {
                    float bp = bpZvar[a][z], pk = pkZvar[a][z], mid = pkMid[a][z];
                    const float nf = (float)pkMidFrames[a][z];
                    const float nb = (float)pkMidBases[a][z];
                    bp = (bp - (mid * mid / nf)) / nf;
                    bp = bp * nb / (nb - 1.0f);
                    const float blVar = blStat.Variance(z);
                    bp -= blVar / (nf / nb);
                    pk = (pk - (mid * mid / nf)) / (nf - 1.0f);
                    pk -= bp + blVar;
                    const float mv = modelVar[a][z];
                    bool mask = mv < blVar;
                    pk /= mv - blVar;
                    mask |= pk < 0.0f;
                    pk = mask ? 0.0f : pk;
                    const float pkm = mid / nf;
                    mask = pkm < 0.0f;
                    bp /= (pkm * pkm);
                    mask |= bp < 0.0f;
                    bp = mask ? kNaN : bp;
                    const int16_t nbi = (int16_t)pkMidBases[a][z];
                    bool m2 = nbi == 0;
                    mid = m2 ? kNaN : mid;
                    m2 |= nbi < 2;
                    m2 |= (int16_t)pkMidFrames[a][z] < 2;
                    bp = m2 ? kNaN : bp;
                    pk = m2 ? kNaN : pk;
                    pkMid[a][z] = mid; bpZvar[a][z] = bp; pkZvar[a][z] = pk;
                }
            }
        }
        FZ
        {
            float s = pdScore[z] / (float)numFrames[z];
            pdScore[z] = std::isnan(s) ? 0.0f : s;
        }
        if (realtime && cart) LabelBlock(frameRate, *cart);
    }

    // LabelBlock, :65-201
    void LabelBlock(float frameRate, const HfCart& cart)
    {
        FZ
        {
            float f[11] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
            const float stdDev = std::sqrt(blStat.Variance(z));
            const float nBases = (float)NumBases(z);
            const float nPulses = (float)NumPulses(z);
            float pw = (float)pulseFrames[z] / nPulses;
            pw = std::isnan(pw) ? 0.0f : pw;
            float pkmid[4];
            for (int a = 0; a < 4; ++a) pkmid[a] = pkMid[a][z] / (float)pkMidFrames[a][z];
            const float seconds = (float)numFrames[z] / frameRate;
            f[0] = nPulses / seconds;
            f[1] = (float)sandwiches[z] / nPulses;
            f[1] = std::isnan(f[1]) ? 0.0f : f[1];
            float hswr = (float)halfSandwiches[z] / nPulses;
            hswr = std::isnan(hswr) ? 0.0f : hswr;
            float hswrExp = cart.hsw[0];
            hswrExp = hswrExp * f[0] + cart.hsw[1];
            hswrExp = (hswrExp > cart.maxHsw) ? cart.maxHsw : hswrExp;
            f[2] = hswr - hswrExp;
            f[3] = pdScore[z];
            f[4] = pw;
            f[5] = (float)stutters[z] / nPulses;
            f[5] = std::isnan(f[5]) ? 0.0f : f[5];
            float rel[4];
            for (int a = 0; a < 4; ++a) rel[a] = modelMean[a][z];
            float maxamp = rel[0];
            for (int a = 1; a < 4; ++a) maxamp = fmax_sse(rel[a], maxamp);
            for (int a = 0; a < 4; ++a) rel[a] /= maxamp;
            unsigned lowIdx = 0;
            float minamp = rel[0];
            for (int a = 1; a < 4; ++a)
            {
                lowIdx = (rel[a] < minamp) ? (unsigned)a : lowIdx;
                minamp = fmin_sse(rel[a], minamp);
            }
            for (int a = 0; a < 4; ++a)
                f[6] += pkmid[a] / stdDev * (float)basesBy[a][z] / nBases * minamp / rel[a];
            f[6] = std::isnan(f[6]) ? 0.0f : f[6];
            for (int a = 0; a < 4; ++a) f[7] = fmax_sse(f[7], (pkMax[a][z] - pkmid[a]) / stdDev);
            f[7] = std::isnan(f[7]) ? 0.0f : f[7];
            f[8] = Autocorrelation(corr, z);
            for (int a = 0; a < 4; ++a)
            {
                float t = bpZvar[a][z];
                f[9] += (std::isnan(t) | (lowIdx == (unsigned)a)) ? 0.0f : t;
                t = pkZvar[a][z];
                f[10] += (std::isnan(t) | (lowIdx == (unsigned)a)) ? 0.0f : t;
            }
            f[9] /= 3.0f;
            f[10] /= 3.0f;
            size_t cur = 0;
            while (cart.feature[cur] >= 0)
                cur = (f[cart.feature[cur]] <= cart.thr[cur]) ? (size_t)cart.left[cur] : (size_t)cart.right[cur];
            activity[z] = (uint8_t)cart.value[cur];
        }
    }

    // PopulateBasecallingMetrics, :203-247
    void Populate(hw_basecalling_metrics& m) const
    {
        FZ
        {
            float ac = Autocorrelation(corr, z);
            ac = std::isnan(ac) ? 0.0f : ac;
            m.activity_label[z] = activity[z];
            m.num_pulse_frames[z] = pulseFrames[z];
            m.num_base_frames[z] = baseFrames[z];
            m.num_sandwiches[z] = sandwiches[z];
            m.num_half_sandwiches[z] = halfSandwiches[z];
            m.num_pulse_label_stutters[z] = stutters[z];
            m.num_bases[z] = NumBases(z);
            m.num_pulses[z] = NumPulses(z);
            for (int a = 0; a < 4; ++a)
            {
                m.pk_mid_signal[a][z] = pkMid[a][z];
                m.bp_zvar[a][z] = bpZvar[a][z];
                m.pk_zvar[a][z] = pkZvar[a][z];
                m.pk_max[a][z] = pkMax[a][z];
                m.num_pk_mid_frames[a][z] = pkMidFrames[a][z];
                m.num_pk_mid_bases_by_analog[a][z] = pkMidBases[a][z];
                m.num_bases_by_analog[a][z] = basesBy[a][z];
                m.num_pulses_by_analog[a][z] = pulsesBy[a][z];
            }
            m.frame_baseline_dws[z] = blStat.Mean(z);
            m.frame_baseline_variance_dws[z] = blStat.Variance(z);
            m.num_frames_baseline[z] = (uint16_t)blStat.m0[z];
            m.start_frame[z] = startFrame[z];
            m.num_frames[z] = (uint16_t)numFrames[z];
            m.autocorrelation[z] = ac;
            m.pulse_detection_score[z] = pdScore[z];
            m.pixel_checksum[z] = pixelChecksum[z];
        }
    }
};

// HFMetricsFilterHost for one pool
struct OracleHf
{
    std::vector<HfLane> lanes;
    uint32_t block = 4096, framesSeen = 0;
    float frameRate = 100.0f;
    bool realtime = true;
    bool haveCart = false;
    HfCart cart;
};

}   // namespace

extern "C" {

void* or_hf_create(uint32_t lanes, uint32_t framesPerBlock, double frameRate, int32_t realtime)
{
    auto* h = new OracleHf;
    h->lanes.resize(lanes);
    for (auto& l : h->lanes) l.Init();
    h->block = framesPerBlock;
    h->frameRate = (float)frameRate;
    h->realtime = realtime != 0;
    return h;
}

void or_hf_destroy(void* p) { delete static_cast<OracleHf*>(p); }

int or_hf_set_cart(void* p, const int16_t* left, const int16_t* right, const int8_t* feature, const float* thr,
                   const int8_t* value, uint32_t n, const float* hsw, float maxHsw)
{
    auto* h = static_cast<OracleHf*>(p);
    h->cart.left.assign(left, left + n);
    h->cart.right.assign(right, right + n);
    h->cart.feature.assign(feature, feature + n);
    h->cart.thr.assign(thr, thr + n);
    h->cart.value.assign(value, value + n);
    h->cart.hsw[0] = hsw[0];
    h->cart.hsw[1] = hsw[1];
    h->cart.maxHsw = maxHsw;
    h->haveCart = true;
    return HW_OK;
}

// HFMetricsFilterHost::Process, :80-118
int or_hf_process(void* p, const hw_pulse* pulses, const uint32_t* lens, uint32_t cap, const hw_baseliner_stats* bs,
                  const hw_lane_model* models, const float* viterbi, const hw_stat_accum_state* pd,
                  int32_t firstFrame, uint32_t frames, hw_basecalling_metrics* out, int32_t* emitted)
{
    auto* h = static_cast<OracleHf*>(p);
    const size_t L = h->lanes.size();
    if (h->framesSeen == 0)
        for (auto& l : h->lanes) l.Reset();
    for (size_t l = 0; l < L; ++l)
    {
        HfLane& m = h->lanes[l];
        m.Count(pulses + l * kLane * cap, lens + l * kLane, cap, frames);
        m.AddModels(models[l]);
        m.AddBatchMetrics(bs[l], viterbi + l * kLane, pd[l]);
    }
    h->framesSeen += frames;
    const uint32_t last = (uint32_t)(firstFrame + (int32_t)frames);
    *emitted = 0;
    if (last % h->block < frames)
    {
        for (size_t l = 0; l < L; ++l)
        {
            h->lanes[l].Finalize(h->realtime, h->frameRate, h->haveCart ? &h->cart : nullptr);
            h->lanes[l].Populate(out[l]);
        }
        h->framesSeen = 0;
        *emitted = 1;
    }
    return HW_OK;
}

}   // extern "C"

// ===========================================================================
// Ingest repacking: appModules/BlockRepacker.cpp:252-345 (BatchFiller::Process),
// every cache line of every packet block copied to its pool / lane / frame.

extern "C" {

int or_repack(uint32_t numZmw, uint32_t lanesPerPool, uint32_t F, int32_t encoding, const hw_sensor_packet* packets,
              uint32_t nPackets, const uint8_t* data, int32_t chunkFirstFrame, uint8_t* const* poolChunks)
{
    const size_t e = encoding == 0 ? 2 : 1;
    const size_t cacheLineZmw = encoding == 0 ? 32 : 64;
    const size_t laneWidth = kLane;
    for (uint32_t i = 0; i < nPackets; ++i)
    {
        const hw_sensor_packet& p = packets[i];
        const size_t W = p.block_width;
        for (size_t blk = 0; blk < p.num_blocks; ++blk)
        {
            const size_t blockZmw = p.start_zmw + blk * W;
            const uint8_t* blockData = data + p.data_offset + blk * p.num_frames * W * e;
            for (size_t f = 0; f < p.num_frames; ++f)
            {
                const size_t batchFrame = (size_t)(p.start_frame - chunkFirstFrame) + f;
                for (size_t zi = 0; zi < W; zi += cacheLineZmw)
                {
                    const size_t zmw = blockZmw + zi;
                    if (zmw >= numZmw) break;
                    const size_t lane = zmw / laneWidth;
                    const size_t pool = lane / lanesPerPool, lip = lane % lanesPerPool;
                    uint8_t* dst = poolChunks[pool] + ((lip * F + batchFrame) * laneWidth + (zmw - lane * laneWidth)) * e;
                    std::memcpy(dst, blockData + (f * W + zi) * e, cacheLineZmw * e);
                }
            }
        }
    }
    return HW_OK;
}

}   // extern "C"

// ===========================================================================
// BAZ pulse encoding: bazio/encoding/ObjectToBaz.h:60-150 (GroupEncoder),
// :373-393 (grouping), FieldSerializers.h:56-364, FieldTransforms.h (NoOp,
// FloatFixedCodec, DeltaCompression), basecaller/dataTypes/PulseFieldAccessors.h
// (field values of a pulse).  The fields are a runtime list here.

namespace {

struct BazPulse          // the field values of one pulse
{
    uint8_t label;
    uint32_t start;
    uint16_t width;
    uint8_t isBase;
    float pkmax, pkmid, pkmean, pkvar;
};

constexpr uint64_t kFfNan = 0, kFfInf = 1, kFfNinf = 2, kFfOffset = 3;

struct BazOracle
{
    std::vector<hw_baz_field> f;
    std::vector<std::vector<int>> groups;      // field indices per group
    std::vector<int> groupBytes;

    explicit BazOracle(const hw_baz_field* fields, uint32_t n) : f(fields, fields + n)
    {
        int cur = 0;
        std::vector<int> g;
        for (uint32_t i = 0; i < n; ++i)
        {
            const int bits = f[i].num_bits;
            const bool even = cur % 8 == 0 && cur > 0;
            if (even || cur + bits > 64)
            {
                groups.push_back(g); groupBytes.push_back((cur + 7) / 8);
                g.clear(); cur = 0;
            }
            g.push_back((int)i); cur += bits;
        }
        groups.push_back(g); groupBytes.push_back((cur + 7) / 8);
    }

    static uint64_t FloatFixed(float v, bool sgn, int scale, int bytes)
    {
        float scaled = std::round(v * (float)scale);
        if (sgn)
        {
            const int64_t mx = (int64_t)((1ull << (8 * bytes - 1)) - 1 - kFfOffset);
            if ((float)(-mx) <= scaled && (float)mx >= scaled)
            {
                if (scaled >= 0) scaled += (float)kFfOffset;
                return (uint64_t)(int64_t)scaled;
            }
        }
        else
        {
            // 8 bytes: the largest code less the offset (a shift by 64 is undefined)
            const uint64_t mx = (bytes >= 8 ? ~0ull : (1ull << (8 * bytes)) - 1) - kFfOffset;
            if (0 <= scaled && (float)mx >= scaled)
            {
                scaled += (float)kFfOffset;
                return (uint64_t)scaled;
            }
        }
        if (std::isnan(v)) return kFfNan;
        if (scaled < 0) return kFfNinf;
        return kFfInf;
    }

    // the transformed value of field i (DeltaCompression updates last[i])
    uint64_t Value(int i, const BazPulse& p, uint64_t* last) const
    {
        const hw_baz_field& d = f[i];
        if (d.transform == HW_BAZ_FLOAT_FIXED)
        {
            const float v = d.name == HW_BAZ_PKMAX ? p.pkmax : d.name == HW_BAZ_PKMID ? p.pkmid
                          : d.name == HW_BAZ_PKMEAN ? p.pkmean : p.pkvar;
            return FloatFixed(v, d.store_signed != 0, d.scale, d.transform_bytes);
        }
        const uint64_t raw = d.name == HW_BAZ_LABEL ? p.label : d.name == HW_BAZ_START_FRAME ? p.start
                           : d.name == HW_BAZ_PULSE_WIDTH ? p.width : p.isBase;
        if (d.transform == HW_BAZ_DELTA)
        {
            const uint64_t r = raw - last[i];
            last[i] = raw;
            return r;
        }
        return raw;
    }

    static bool SimpleNeeds(uint64_t v, bool sgn, int bits)
    {
        if (sgn) v += (1ull << (bits - 1)) - 1;
        return v >= (1ull << bits) - 1;
    }

    static size_t CompactOverflowBytes(uint64_t t, bool sgn, int bits)
    {
        if (sgn)
        {
            const int discard = __builtin_clrsbl((long)t);
            const int keep = 64 - discard - (bits - 1);
            return (size_t)((keep + 6) / 7);
        }
        t >>= (bits - 1);
        size_t r = 0;
        while (t) { ++r; t >>= 7; }
        return r;
    }

    size_t OverflowBytes(int i, uint64_t v) const
    {
        const hw_baz_field& d = f[i];
        if (d.serialize == HW_BAZ_SIMPLE_OVERFLOW)
            return SimpleNeeds(v, d.store_signed != 0, d.num_bits) ? (size_t)d.overflow_bytes : 0;
        if (d.serialize == HW_BAZ_COMPACT_OVERFLOW) return CompactOverflowBytes(v, d.store_signed != 0, d.num_bits);
        return 0;
    }

    uint64_t ToBinary(int i, uint64_t v, uint8_t*& ptr) const
    {
        const hw_baz_field& d = f[i];
        const int bits = d.num_bits;
        if (d.serialize == HW_BAZ_SIMPLE_OVERFLOW)
        {
            if (SimpleNeeds(v, d.store_signed != 0, bits))
            {
                std::memcpy(ptr, &v, (size_t)d.overflow_bytes);
                ptr += d.overflow_bytes;
                return (1ull << bits) - 1;
            }
            if (d.store_signed) v += (1ull << (bits - 1)) - 1;
            return v;
        }
        if (d.serialize == HW_BAZ_COMPACT_OVERFLOW)
        {
            const uint64_t cmask = 1ull << (bits - 1), vmask = cmask - 1;
            size_t n = CompactOverflowBytes(v, d.store_signed != 0, bits);
            uint64_t first = v & vmask;
            v >>= (bits - 1);
            if (n) first |= cmask;
            while (n)
            {
                uint8_t b = (uint8_t)(v & 0x7f);
                v >>= 7;
                --n;
                if (n) b |= 0x80;
                *ptr++ = b;
            }
            return first;
        }
        return v;
    }

    // BytesRequired + Serialize of one pulse (PacketBuffer::AddZmw)
    size_t Bytes(const BazPulse& p, uint64_t* last) const
    {
        size_t n = 0;
        for (size_t g = 0; g < groups.size(); ++g)
        {
            n += (size_t)groupBytes[g];
            for (int i : groups[g]) n += OverflowBytes(i, Value(i, p, last));
        }
        return n;
    }

    uint8_t* Encode(const BazPulse& p, uint8_t* ptr, uint64_t* last) const
    {
        for (size_t g = 0; g < groups.size(); ++g)
        {
            uint64_t data = 0;
            uint8_t* ptr2 = ptr + groupBytes[g];
            size_t pos = 0;
            for (int i : groups[g])
            {
                const int bits = f[i].num_bits;
                const uint64_t v = ToBinary(i, Value(i, p, last), ptr2);
                data |= (v & (uint64_t)((1 << bits) - 1)) << pos;
                pos += (size_t)bits;
            }
            std::memcpy(ptr, &data, (size_t)groupBytes[g]);
            ptr = ptr2;
        }
        return ptr;
    }

    // FieldSerializers.h FromBinary: the main bits `val` plus overflow bytes at ptr
    uint64_t FromBinary(int i, uint64_t val, const uint8_t*& ptr) const
    {
        const hw_baz_field& d = f[i];
        const int bits = d.num_bits;
        const bool sgn = d.store_signed != 0;
        uint64_t ret = val;
        if (d.serialize == HW_BAZ_TRUNCATE)
        {
            if (sgn && (val & (1ull << (bits - 1)))) ret |= (~0ull << bits);
        }
        else if (d.serialize == HW_BAZ_SIMPLE_OVERFLOW)
        {
            if (val == (1ull << bits) - 1)
            {
                ret = 0;
                std::memcpy(&ret, ptr, (size_t)d.overflow_bytes);
                ptr += d.overflow_bytes;
                const int sb = 8 * d.overflow_bytes;
                if (sgn && (ret & (1ull << (sb - 1)))) ret |= (~0ull << (sb - 1));
            }
            else if (sgn) ret = val - ((1ull << (bits - 1)) - 1);
        }
        else
        {
            const uint64_t cmask = 1ull << (bits - 1);
            ret = val & (cmask - 1);
            bool cont = (val & cmask) != 0;
            int cur = bits - 1;
            while (cont)
            {
                const uint64_t b = *ptr++;
                cont = (b & 0x80) != 0;
                ret |= (b & 0x7f) << cur;
                cur += 7;
            }
            if (sgn && (ret & (1ull << (cur - 1)))) ret |= ~0ull << cur;
        }
        return ret;
    }

    // FloatFixedCodec::Revert
    static float FloatFixedRevert(uint64_t ret, bool sgn, int scale)
    {
        if (ret == kFfNan) return kNaN;
        if (ret == kFfInf) return std::numeric_limits<float>::infinity();
        if (ret == kFfNinf) return -std::numeric_limits<float>::infinity();
        if (sgn)
        {
            int64_t s = (int64_t)ret;
            if (s >= 0) s -= (int64_t)kFfOffset;
            return (float)s / (float)scale;
        }
        return (float)(ret - kFfOffset) / (float)scale;
    }

    // Decode (for round trips)
    const uint8_t* Decode(const uint8_t* ptr, BazPulse& p, uint64_t* last) const
    {
        for (size_t g = 0; g < groups.size(); ++g)
        {
            uint64_t data = 0;
            std::memcpy(&data, ptr, (size_t)groupBytes[g]);
            ptr += groupBytes[g];
            for (int i : groups[g])
            {
                const hw_baz_field& d = f[i];
                const int bits = d.num_bits;
                const uint64_t val = data & (uint64_t)((1 << bits) - 1);
                data >>= bits;
                uint64_t ret = FromBinary(i, val, ptr);
                // the transforms' Revert
                if (d.transform == HW_BAZ_DELTA) { last[i] += ret; ret = last[i]; }
                if (d.transform == HW_BAZ_FLOAT_FIXED)
                {
                    const float fv = FloatFixedRevert(ret, d.store_signed != 0, d.scale);
                    if (d.name == HW_BAZ_PKMAX) p.pkmax = fv;
                    else if (d.name == HW_BAZ_PKMID) p.pkmid = fv;
                    else if (d.name == HW_BAZ_PKMEAN) p.pkmean = fv;
                    else p.pkvar = fv;
                    continue;
                }
                if (d.name == HW_BAZ_LABEL) p.label = (uint8_t)ret;
                else if (d.name == HW_BAZ_START_FRAME) p.start = (uint32_t)ret;
                else if (d.name == HW_BAZ_PULSE_WIDTH) p.width = (uint16_t)ret;
                else p.isBase = (uint8_t)ret;
            }
        }
        return ptr;
    }
};

// PulseFieldAccessors.h:43-68 on the basecaller's Pulse (signals in 0.1 DN steps)
BazPulse FromHwPulse(const hw_pulse& p)
{
    BazPulse b;
    b.label = p.label;
    b.start = p.start;
    b.width = p.width;
    b.isBase = p.is_reject ? 0 : 1;
    b.pkmax = (float)p.max_signal * 0.1f;
    b.pkmid = p.width < 3 ? kNaN : (float)p.mid_signal * 0.1f;
    b.pkmean = (float)p.mean_signal * 0.1f;
    b.pkvar = p.width < 3 ? kNaN : p.signal_m2;
    return b;
}

}   // namespace

extern "C" {

// One serializer alone (FieldSerializers.h): ToBinary of val, the main bits
// masked to num_bits when mask is set, then FromBinary.  *overflow receives
// OverflowBytes(val); the return value is the decoded value.
uint64_t or_baz_serializer_roundtrip(int32_t serialize, int32_t numBits, int32_t overflowBytes, int32_t sgn,
                                     uint64_t val, int32_t mask, uint64_t* overflow)
{
    hw_baz_field d{};
    d.serialize = serialize;
    d.num_bits = numBits;
    d.overflow_bytes = overflowBytes;
    d.store_signed = sgn;
    BazOracle o(&d, 1);
    *overflow = o.OverflowBytes(0, val);
    uint8_t buf[16] = {};
    uint8_t* w = buf;
    uint64_t main = o.ToBinary(0, val, w);
    if (mask) main &= (1ull << numBits) - 1;
    const uint8_t* r = buf;
    return o.FromBinary(0, main, r);
}

// FloatFixedCodec Apply then Revert; *code receives the transformed value.
float or_baz_float_fixed_roundtrip(float v, int32_t sgn, int32_t scale, int32_t bytes, uint64_t* code)
{
    *code = BazOracle::FloatFixed(v, sgn != 0, scale, bytes);
    return BazOracle::FloatFixedRevert(*code, sgn != 0, scale);
}

// One ZMW's pulse sequence (field values), encoded with `last` (one uint64 per
// field) carried in and out.  Returns the byte count; writes at most cap.
int64_t or_baz_encode_values(const hw_baz_field* fields, uint32_t nf, const void* pulses, uint32_t n, uint8_t* out,
                             uint64_t cap, uint64_t* last)
{
    BazOracle o(fields, nf);
    const BazPulse* p = static_cast<const BazPulse*>(pulses);
    std::vector<uint64_t> copy(last, last + nf);
    size_t need = 0;
    for (uint32_t i = 0; i < n; ++i) need += o.Bytes(p[i], copy.data());
    if (need > cap) return -1;
    uint8_t* ptr = out;
    for (uint32_t i = 0; i < n; ++i) ptr = o.Encode(p[i], ptr, last);
    return (int64_t)(ptr - out);
}

int or_baz_decode_values(const hw_baz_field* fields, uint32_t nf, const uint8_t* bytes, uint32_t n, void* pulses,
                         uint64_t* last, uint64_t* consumed)
{
    BazOracle o(fields, nf);
    BazPulse* p = static_cast<BazPulse*>(pulses);
    const uint8_t* ptr = bytes;
    for (uint32_t i = 0; i < n; ++i)
    {
        p[i] = BazPulse{};
        ptr = o.Decode(ptr, p[i], last);
    }
    *consumed = (uint64_t)(ptr - bytes);
    return HW_OK;
}

// PrelimHQFilter + PacketBuffer::AddZmw over a chunk of the basecaller's
// pulses: per ZMW the kept pulses in order, bytes appended to out;
// offsets[numZmw + 1].  last[numZmw][nf] carries the delta state.
// zmwStride: only ZMW 0, stride, 2 x stride ... of each lane of 64
// (PrelimHQFilter.cpp:107-118).
int or_baz_encode_chunk(const hw_baz_field* fields, uint32_t nf, int32_t skipRejects, uint32_t numZmw,
                        uint32_t zmwStride, const hw_pulse* pulses, const uint32_t* lens, uint32_t cap, uint8_t* out,
                        uint64_t outCap, uint64_t* offsets, uint64_t* last)
{
    BazOracle o(fields, nf);
    uint64_t pos = 0;
    for (uint32_t z = 0; z < numZmw; ++z)
    {
        offsets[z] = pos;
        if ((z % 64) % zmwStride != 0) continue;
        const uint32_t n = std::min(lens[z], cap);
        for (uint32_t i = 0; i < n; ++i)
        {
            const hw_pulse& hp = pulses[(size_t)z * cap + i];
            if (skipRejects && hp.is_reject) continue;
            const BazPulse b = FromHwPulse(hp);
            std::vector<uint64_t> copy(last + (size_t)z * nf, last + (size_t)(z + 1) * nf);
            const size_t need = o.Bytes(b, copy.data());
            if (pos + need > outCap) return HW_ERR_OUT_OF_MEMORY;
            uint8_t* end = o.Encode(b, out + pos, last + (size_t)z * nf);
            pos = (uint64_t)(end - out);
        }
    }
    offsets[numZmw] = pos;
    return HW_OK;
}

}   // extern "C"

// ---- Preliminary HQ stage -------------------------------------------------------
// bazio/writing/PacketBufferManager.cpp:43-176 (what a checkpoint holds for
// each ZMW: nothing while it is pre-HQ, its data of the current metric block
// once HQ, and on the block it is marked HQ every block of the lookback
// window, oldest first; data older than the window is dropped) and
// basecaller/appModules/PrelimHQFilter.cpp:133-215 (DetectHQ: every ZMW marked
// HQ when the preliminary HQ step is off; otherwise, from the lookbackSize-th
// metric block on, every round(1/hqThrottleFraction)-th ZMW still pre-HQ, in
// ZMW order).  Each ZMW keeps a list of per-block (bytes, events), the
// current block last.

namespace {

struct PreHqOracle
{
    uint32_t numZmw, lookback;
    bool enable;
    size_t stride;
    size_t seen = 0;
    std::vector<uint8_t> hq;
    std::vector<std::deque<std::pair<std::vector<uint8_t>, uint32_t>>> blocks;

    PreHqOracle(uint32_t n, uint32_t lb, bool en, float throttle)
        : numZmw(n), lookback(lb), enable(en), stride((size_t)std::round(1 / throttle)), hq(n, 0), blocks(n)
    {
        for (auto& d : blocks) d.emplace_back();
    }

    void Add(const uint8_t* bytes, const uint64_t* offsets, const uint32_t* events)
    {
        for (uint32_t z = 0; z < numZmw; ++z)
        {
            auto& b = blocks[z].back();
            b.first.insert(b.first.end(), bytes + offsets[z], bytes + offsets[z + 1]);
            b.second += events[z];
        }
    }

    // the ZMWs newly HQ at this block's end
    std::vector<uint8_t> Mark(const uint8_t* marks)
    {
        std::vector<uint8_t> newly(numZmw, 0);
        if (marks)
        {
            for (uint32_t z = 0; z < numZmw; ++z) newly[z] = !hq[z] && marks[z];
            ++seen;
            return newly;
        }
        if (!enable)
        {
            for (uint32_t z = 0; z < numZmw; ++z) newly[z] = !hq[z];
            return newly;
        }
        if (++seen < lookback) return newly;
        size_t counter = 0;
        for (uint32_t z = 0; z < numZmw; ++z)
        {
            if (hq[z]) continue;
            if (counter % stride == 0) newly[z] = 1;
            ++counter;
        }
        return newly;
    }

    // the checkpoint's bytes; false when they pass cap (nothing changes then)
    int64_t Output(const std::vector<uint8_t>& newly, bool flush, uint8_t* out, uint64_t cap, uint64_t* offsets,
                   uint32_t* events, uint8_t* hqOut)
    {
        uint64_t pos = 0;
        std::vector<std::pair<uint64_t, uint32_t>> sizes(numZmw);
        for (uint32_t z = 0; z < numZmw; ++z)
        {
            uint64_t n = 0;
            uint32_t ev = 0;
            if (hq[z])
            {
                n = blocks[z].back().first.size();
                ev = blocks[z].back().second;
            }
            else if (!flush && newly[z])
                for (const auto& b : blocks[z])
                {
                    n += b.first.size();
                    ev += b.second;
                }
            sizes[z] = {n, ev};
            pos += n;
        }
        if (pos > cap) return -1;
        pos = 0;
        for (uint32_t z = 0; z < numZmw; ++z)
        {
            offsets[z] = pos;
            events[z] = sizes[z].second;
            if (hq[z] || (!flush && newly[z]))
            {
                const size_t from = hq[z] ? blocks[z].size() - 1 : 0;
                for (size_t i = from; i < blocks[z].size(); ++i)
                {
                    const auto& b = blocks[z][i].first;
                    std::copy(b.begin(), b.end(), out + pos);
                    pos += b.size();
                }
            }
        }
        offsets[numZmw] = pos;
        if (!flush)
            for (uint32_t z = 0; z < numZmw; ++z)
            {
                if (hq[z] || newly[z])
                {
                    hq[z] = 1;
                    blocks[z].clear();
                }
                blocks[z].emplace_back();
                if (blocks[z].size() > lookback) blocks[z].pop_front();
            }
        for (uint32_t z = 0; z < numZmw; ++z) hqOut[z] = hq[z];
        return (int64_t)pos;
    }
};

}   // namespace

extern "C" {

void* or_prehq_create(uint32_t numZmw, uint32_t lookback, int32_t enable, float throttle)
{
    return new PreHqOracle(numZmw, lookback, enable != 0, throttle);
}

void or_prehq_destroy(void* h) { delete static_cast<PreHqOracle*>(h); }

void or_prehq_add(void* h, const uint8_t* bytes, const uint64_t* offsets, const uint32_t* events)
{
    static_cast<PreHqOracle*>(h)->Add(bytes, offsets, events);
}

// End of a metric block: marks (the placeholder rule, or `marks` when not
// null), then the checkpoint.  Returns its bytes, or -1 when they pass cap
// (the marks are then discarded and nothing changes).
int64_t or_prehq_end_block(void* h, const uint8_t* marks, uint8_t* out, uint64_t cap, uint64_t* offsets,
                           uint32_t* events, uint8_t* hq)
{
    auto* o = static_cast<PreHqOracle*>(h);
    const size_t seen = o->seen;
    const auto newly = o->Mark(marks);
    const int64_t n = o->Output(newly, false, out, cap, offsets, events, hq);
    if (n < 0) o->seen = seen;
    return n;
}

int64_t or_prehq_flush(void* h, uint8_t* out, uint64_t cap, uint64_t* offsets, uint32_t* events, uint8_t* hq)
{
    auto* o = static_cast<PreHqOracle*>(h);
    return o->Output(std::vector<uint8_t>(o->numZmw, 0), true, out, cap, offsets, events, hq);
}

}   // extern "C"

// ---- Metric side of the preliminary HQ stage ------------------------------------
// basecaller/dataTypes/Metrics.h:36-366 (ProductionMetrics and
// CompleteMetrics: construction from BasecallingMetrics :53-70 / :212-228,
// Aggregate :73-118 / :230-286, Convert :121-146 / :288-318) and
// bazio/writing/MetricBufferManager.h:70-357 (AddZmw, MarkAsHQ, Flush,
// UpdateLookback, AddProductionMetrics, NumTransitionsInLookbackWindow,
// AddLookbackWindowMetricBlocks), restated over the same data structures: a
// window of per-block buffers whose entries are linked by next-buffer
// indices, per-ZMW (hqStarted, currentIndex, recentIndex) and one open
// aggregate per ZMW.  AddZmw is called for ZMWs z with z % stride == 0
// (PrelimHQFilter.cpp:107-118); entries never written read as
// default-constructed blocks (the reference reads uninitialised memory
// there), and a newly-HQ ZMW whose window holds fewer label runs than blocks
// it writes keeps only the first NumTransitions of them (the reference
// writes the rest past the end of its output view).
//
// Two index slips of the reference are kept apart under `literal`:
// AddProductionMetrics aggregates an HQ ZMW into the open aggregate at its
// stale window index instead of its own (MetricBufferManager.h:263), and
// AddLookbackWindowMetricBlocks reads each buffer after the front at the
// index of the buffer before it (:318, the index advances after the read).
// Both are no-ops while no ZMW below the one concerned was marked HQ in the
// blocks its indices span; past that the reference reads other ZMWs'
// entries and, where its index runs past a buffer or through an entry that
// was never linked, memory it never wrote (read here as a default block and
// index 0).  With `literal` off the oracle follows each ZMW's own entries
// and aggregate, which is what the stage computes.
//
// The half type is the `half` library 2.1.0 (half.sourceforge.net; pinned by
// basecaller/nexus-versions/Fetchhalf.cmake:3 and not in the reference tree):
// float -> half rounds to nearest with ties to even (its default round
// style), half -> float is exact, and half sqrt is correctly rounded, which
// equals rounding the correctly-rounded float sqrt to half (24 >= 2*11 + 2
// bits).  NaN converts to the quiet NaN 0x7fff / 0xffff.

namespace {

uint16_t HalfBits(float f)
{
    uint32_t x;
    std::memcpy(&x, &f, 4);
    const uint16_t sign = (uint16_t)((x >> 16) & 0x8000u);
    const uint32_t ax = x & 0x7fffffffu;
    if (ax > 0x7f800000u) return (uint16_t)(sign | 0x7fffu);    // NaN
    if (ax >= 0x477ff000u) return (uint16_t)(sign | 0x7c00u);   // >= 65520 (and inf) -> inf
    if (ax < 0x38800000u)                                        // below 2^-14: subnormal or zero
    {
        const int e = (int)(ax >> 23);
        const int shift = 126 - e;                               // value = m * 2^(e-150); unit 2^-24
        if (shift > 24) return sign;
        const uint32_t m = (ax & 0x7fffffu) | 0x800000u;
        uint32_t h = m >> shift;
        const uint32_t rem = m & ((1u << shift) - 1u), half = 1u << (shift - 1);
        if (rem > half || (rem == half && (h & 1u))) ++h;
        return (uint16_t)(sign | h);
    }
    uint32_t h = (ax - 0x38000000u) >> 13;                       // rebias 127 -> 15
    const uint32_t rem = ax & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) ++h;
    return (uint16_t)(sign | h);
}

float HalfFloat(uint16_t h)
{
    const uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    const uint32_t e = (h >> 10) & 0x1fu, m = h & 0x3ffu;
    uint32_t x;
    if (e == 0x1f) x = sign | 0x7f800000u | (m << 13);
    else if (e) x = sign | ((e + 112u) << 23) | (m << 13);
    else if (!m) x = sign;
    else
    {
        int k = 0;
        uint32_t mm = m;
        while (!(mm & 0x400u)) { mm <<= 1; ++k; }
        x = sign | ((uint32_t)(113 - k) << 23) | ((mm & 0x3ffu) << 13);
    }
    float f;
    std::memcpy(&f, &x, 4);
    return f;
}

struct Half
{
    uint16_t bits = 0;
    Half() = default;
    Half(float f) : bits(HalfBits(f)) {}
    operator float() const { return HalfFloat(bits); }
};

float SqrtOf(float v) { return std::sqrt(v); }
float SqrtOf(Half v) { return Half(std::sqrt((float)v)); }

constexpr uint8_t kNoLabel = 4;   // HQRFPhysicalStates::NUM_PHYS_STATES

template <typename U, typename F>
struct ProdBlock
{
    U numFrames = 0, pulseWidth = 0, baseWidth = 0, numPulses = 0, numBases = 0;
    F pkmid[4] = {F(0.f), F(0.f), F(0.f), F(0.f)};
    U numPkmidFrames[4] = {0, 0, 0, 0};
    U numBasesByAnalog[4] = {0, 0, 0, 0};
    F baselineVar = F(0.f), baselineMean = F(0.f);
    U numBaselineFrames = 0;
    uint8_t label = kNoLabel;

    ProdBlock() = default;
    ProdBlock(const hw_basecalling_metrics& bm, int z)
        : numFrames(bm.num_frames[z]), pulseWidth(bm.num_pulse_frames[z]), baseWidth(bm.num_base_frames[z]),
          numPulses(bm.num_pulses[z]), numBases(bm.num_bases[z]), baselineVar(F(bm.frame_baseline_variance_dws[z])),
          baselineMean(F(bm.frame_baseline_dws[z])), numBaselineFrames(bm.num_frames_baseline[z]),
          label(bm.activity_label[z])
    {
        for (int a = 0; a < 4; ++a)
        {
            numPkmidFrames[a] = bm.num_pk_mid_frames[a][z];
            const float v = numPkmidFrames[a] > 0 ? bm.pk_mid_signal[a][z] / (float)numPkmidFrames[a] : 0.0f;
            pkmid[a] = F(v);
            numBasesByAnalog[a] = bm.num_bases_by_analog[a][z];
        }
    }

    bool HasData() const { return numFrames != 0; }

    // Metrics.h:73-118, every product and sum in float
    template <typename U2, typename F2>
    void Aggregate(const ProdBlock<U2, F2>& b)
    {
        const U nbf = (U)(numBaselineFrames + b.numBaselineFrames);
        float mean = (float)numBaselineFrames * (float)baselineMean;
        mean = mean + (float)b.numBaselineFrames * (float)b.baselineMean;
        baselineMean = F(mean);
        if (nbf > 0)
        {
            baselineMean = F((float)baselineMean / (float)nbf);
            float bv = 0.0f;
            U nk = nbf;
            auto pooled = [&](uint64_t n0, float var) {
                const uint64_t n = n0 > 1 ? n0 - 1 : n0;
                bv = bv + (float)n * var;
                return n0 > 0;
            };
            if (pooled(numBaselineFrames, (float)baselineVar)) --nk;
            if (pooled(b.numBaselineFrames, (float)b.baselineVar)) --nk;
            baselineVar = F(bv / (float)nk);
            numBaselineFrames = nbf;
        }
        for (int a = 0; a < 4; ++a)
        {
            float p = (float)numPkmidFrames[a] * (float)pkmid[a];
            p = p + (float)b.numPkmidFrames[a] * (float)b.pkmid[a];
            numPkmidFrames[a] = (U)(numPkmidFrames[a] + b.numPkmidFrames[a]);
            if (numPkmidFrames[a] > 0) p = p / (float)numPkmidFrames[a];
            pkmid[a] = F(p);
            numBasesByAnalog[a] = (U)(numBasesByAnalog[a] + b.numBasesByAnalog[a]);
        }
        numFrames = (U)(numFrames + b.numFrames);
        pulseWidth = (U)(pulseWidth + b.pulseWidth);
        baseWidth = (U)(baseWidth + b.baseWidth);
        numPulses = (U)(numPulses + b.numPulses);
        numBases = (U)(numBases + b.numBases);
        label = b.label;
    }

    // Metrics.h:121-146 through the uint16_t setters of bazio/MetricBlock.h
    void Convert(hw_spider_metric_block& sm) const
    {
        sm.num_frames = (uint16_t)numFrames;
        sm.pulse_width = (uint16_t)pulseWidth;
        sm.base_width = (uint16_t)baseWidth;
        sm.num_pulses = (uint16_t)numPulses;
        for (int a = 0; a < 4; ++a)
        {
            sm.pkmid[a] = (float)pkmid[a];
            sm.num_pkmid_frames[a] = (uint16_t)numPkmidFrames[a];
            sm.num_bases[a] = (uint16_t)numBasesByAnalog[a];
        }
        sm.baseline = (float)baselineMean;
        sm.baseline_sd = (float)SqrtOf(baselineVar);
        sm.num_baseline_frames = (uint32_t)numBaselineFrames;
        sm.activity_label = label;
    }
};

template <typename U, typename F>
struct CompleteBlock
{
    ProdBlock<U, F> prod;
    U numHalfSandwiches = 0, numSandwiches = 0, numPulseLabelStutters = 0;
    F pulseDetectionScore = F(0.f), traceAutoCorrelation = F(0.f);
    F pkmax[4] = {F(0.f), F(0.f), F(0.f), F(0.f)};
    U numPkmidBases[4] = {0, 0, 0, 0};
    F bpzvar[4] = {F(0.f), F(0.f), F(0.f), F(0.f)};
    F pkzvar[4] = {F(0.f), F(0.f), F(0.f), F(0.f)};

    CompleteBlock() = default;
    CompleteBlock(const hw_basecalling_metrics& bm, int z)
        : prod(bm, z), numHalfSandwiches(bm.num_half_sandwiches[z]), numSandwiches(bm.num_sandwiches[z]),
          numPulseLabelStutters(bm.num_pulse_label_stutters[z]), pulseDetectionScore(F(bm.pulse_detection_score[z])),
          traceAutoCorrelation(F(bm.autocorrelation[z]))
    {
        for (int a = 0; a < 4; ++a)
        {
            pkmax[a] = F(bm.pk_max[a][z]);
            numPkmidBases[a] = bm.num_pk_mid_bases_by_analog[a][z];
            bpzvar[a] = F(bm.bp_zvar[a][z]);
            pkzvar[a] = F(bm.pk_zvar[a][z]);
        }
    }

    // Metrics.h:230-286 (only the reference's own known-answer test
    // aggregates complete metrics; the stage converts them as they arrive)
    template <typename U2, typename F2>
    void Aggregate(const CompleteBlock<U2, F2>& b)
    {
        numHalfSandwiches = (U)(numHalfSandwiches + b.numHalfSandwiches);
        numSandwiches = (U)(numSandwiches + b.numSandwiches);
        numPulseLabelStutters = (U)(numPulseLabelStutters + b.numPulseLabelStutters);
        float pk[4], pkz[4] = {0, 0, 0, 0}, bpz[4] = {0, 0, 0, 0};
        U npf[4], npb[4];
        for (int a = 0; a < 4; ++a)
        {
            const float pa = (float)prod.pkmid[a], pb = (float)b.prod.pkmid[a];
            pk[a] = (float)prod.numPkmidFrames[a] * pa + (float)b.prod.numPkmidFrames[a] * pb;
            npf[a] = (U)(prod.numPkmidFrames[a] + b.prod.numPkmidFrames[a]);
            if (npf[a] > 0) pk[a] = pk[a] / (float)npf[a];
            if (prod.numPkmidFrames[a] > 1) pkz[a] = pkz[a] + (float)prod.numPkmidFrames[a] * (float)pkzvar[a];
            if (b.prod.numPkmidFrames[a] > 1) pkz[a] = pkz[a] + (float)b.prod.numPkmidFrames[a] * (float)b.pkzvar[a];
            npb[a] = (U)(numPkmidBases[a] + b.numPkmidBases[a]);
            if (numPkmidBases[a] > 1) bpz[a] = bpz[a] + (float)bpzvar[a] * pa * pa * (float)numPkmidBases[a];
            if (b.numPkmidBases[a] > 1) bpz[a] = bpz[a] + (float)b.bpzvar[a] * pb * pb * (float)b.numPkmidBases[a];
        }
        for (int a = 0; a < 4; ++a)
        {
            float v = pkz[a];
            if (npf[a] > 1) v = v / (float)npf[a];
            pkzvar[a] = F(v);
            float w = bpz[a];
            numPkmidBases[a] = npb[a];
            if (npf[a] > 0 && numPkmidBases[a] > 1) w = w / ((float)numPkmidBases[a] * pk[a] * pk[a]);
            bpzvar[a] = F(w);
            pkmax[a] = F(std::max((float)pkmax[a], (float)b.pkmax[a]));
        }
        const U nf = (U)(prod.numFrames + b.prod.numFrames);
        float pds = (float)prod.numFrames * (float)pulseDetectionScore + (float)b.prod.numFrames * (float)b.pulseDetectionScore;
        float tac = (float)prod.numFrames * (float)traceAutoCorrelation + (float)b.prod.numFrames * (float)b.traceAutoCorrelation;
        if (nf > 0)
        {
            pds = pds / (float)nf;
            tac = tac / (float)nf;
        }
        pulseDetectionScore = F(pds);
        traceAutoCorrelation = F(tac);
        prod.Aggregate(b.prod);
    }

    void Convert(hw_spider_metric_block& sm) const
    {
        prod.Convert(sm);
        sm.num_half_sandwiches = (uint16_t)numHalfSandwiches;
        sm.num_sandwiches = (uint16_t)numSandwiches;
        sm.num_pulse_label_stutters = (uint16_t)numPulseLabelStutters;
        sm.pulse_detection_score = (float)pulseDetectionScore;
        sm.trace_autocorr = (float)traceAutoCorrelation;
        for (int a = 0; a < 4; ++a)
        {
            sm.pkmax[a] = (float)pkmax[a];
            sm.num_pkmid_bases[a] = (uint16_t)numPkmidBases[a];
            sm.bpzvar[a] = (float)bpzvar[a];
            sm.pkzvar[a] = (float)pkzvar[a];
        }
    }
};

hw_spider_metric_block EmptySpider()
{
    hw_spider_metric_block sm;
    std::memset(&sm, 0, sizeof(sm));
    return sm;
}

// MetricBufferManager over ProductionMetricsGroup (preliminary HQ on) or
// CompleteMetricsGroup (off).
struct MetricSideOracle
{
    using MetricT = ProdBlock<uint16_t, Half>;
    using AggT = ProdBlock<uint32_t, float>;
    struct Buffer
    {
        std::vector<MetricT> data;
        std::vector<uint32_t> next;
        explicit Buffer(size_t n) : data(n), next(n, 0) {}
    };
    struct Info
    {
        bool hqStarted = false;
        uint32_t current = 0, recent = 0;
    };

    uint32_t numZmw, maxLookBack, stride;
    bool production, literal;
    std::vector<uint8_t> recentLabel;
    std::vector<Info> info;
    std::vector<uint8_t> newHq;
    size_t numHq = 0;
    std::vector<AggT> agg;
    std::deque<Buffer> window;
    std::vector<std::vector<hw_spider_metric_block>> out;

    MetricSideOracle(uint32_t n, uint32_t lookback, bool prehq, uint32_t zmwStride, bool lit)
        : numZmw(n), maxLookBack(lookback), stride(zmwStride), production(prehq), literal(lit),
          recentLabel(n, kNoLabel), info(n), newHq(n, 0), agg(n), out(n)
    {
        for (uint32_t z = 0; z < n; ++z) info[z].current = info[z].recent = z;
        if (production) window.emplace_back(n);
    }

    // MetricBufferManager.h:142-149, 240-287
    void AddZmw(uint32_t z, const hw_basecalling_metrics& bm, int lz)
    {
        recentLabel[z] = bm.activity_label[lz];
        if (!production)
        {
            hw_spider_metric_block sm = EmptySpider();
            CompleteBlock<uint16_t, Half>(bm, lz).Convert(sm);
            out[z] = {sm};
            return;
        }
        const MetricT m(bm, lz);
        if (!info[z].hqStarted)
        {
            window.back().data[info[z].recent] = m;
            return;
        }
        AggT& a = agg[literal ? info[z].current : z];
        if (m.label == a.label)
        {
            a.Aggregate(m);
            return;
        }
        if (a.label != kNoLabel)
        {
            hw_spider_metric_block sm = EmptySpider();
            a.Convert(sm);
            out[z] = {sm};
        }
        a = AggT();
        a.Aggregate(m);
    }

    void Add(const hw_basecalling_metrics* lanes)
    {
        for (uint32_t z = 0; z < numZmw; z += stride) AddZmw(z, lanes[z / HW_LANE_SIZE], (int)(z % HW_LANE_SIZE));
    }

    // MetricBufferManager.h:151-159
    void MarkAsHq(uint32_t z)
    {
        if (!production || info[z].hqStarted || newHq[z]) return;
        ++numHq;
        newHq[z] = 1;
    }

    // MetricBufferManager.h:289-305
    size_t Transitions(uint32_t z) const
    {
        uint32_t idx = info[z].current;
        size_t n = 0;
        uint8_t cur = kNoLabel;
        for (const Buffer& b : window)
        {
            const MetricT& m = b.data[idx];
            if (m.label != cur)
            {
                ++n;
                cur = m.label;
            }
            idx = b.next[idx];
        }
        return n;
    }

    // MetricBufferManager.h:180-233 with :307-333
    void UpdateLookback()
    {
        if (!production) return;
        uint32_t lookbackIdx = 0;
        for (uint32_t z = 0; z < numZmw; ++z)
        {
            Info& in = info[z];
            if (in.hqStarted || newHq[z])
            {
                in.hqStarted = true;
                if (!newHq[z]) continue;
                const size_t n = Transitions(z);
                std::vector<hw_spider_metric_block> o(n, EmptySpider());
                auto put = [&](size_t i, const AggT& a) {
                    if (i < n) a.Convert(o[i]);
                };
                put(0, agg[z]);
                uint32_t idx = in.current;
                const MetricT& front = window.front().data[idx];
                uint8_t cur = front.label;
                AggT amb;
                amb.Aggregate(front);
                size_t k = 1;
                for (size_t w = 1; w < window.size(); ++w)
                {
                    const Buffer& b = window[w];
                    MetricT mb;
                    if (literal)
                    {
                        if (idx < b.data.size()) mb = b.data[idx];
                        idx = idx < b.next.size() ? b.next[idx] : 0;
                    }
                    else
                    {
                        idx = window[w - 1].next[idx];
                        mb = b.data[idx];
                    }
                    if (mb.label != cur)
                    {
                        put(k++, amb);
                        cur = mb.label;
                        amb = AggT();
                    }
                    amb.Aggregate(mb);
                }
                out[z] = std::move(o);
                agg[z] = AggT();
                agg[z].Aggregate(amb);
            }
            else
            {
                window.back().next[in.recent] = lookbackIdx;
                in.recent = lookbackIdx++;
                if (window.size() == maxLookBack)
                {
                    const Buffer& f = window.front();
                    agg[z].Aggregate(f.data[in.current]);
                    in.current = f.next[in.current];
                }
            }
        }
        if (maxLookBack > 0)
        {
            window.emplace_back(numZmw - numHq);
            if (window.size() > maxLookBack) window.pop_front();
        }
        std::fill(newHq.begin(), newHq.end(), 0);
    }

    // MetricBufferManager.h:161-178
    void Flush()
    {
        if (!production) return;
        for (uint32_t z = 0; z < numZmw; ++z)
            if (agg[z].HasData())
            {
                hw_spider_metric_block sm = EmptySpider();
                agg[z].Convert(sm);
                out[z] = {sm};
            }
    }

    // GetMetrics; -1 (nothing taken) when the blocks pass cap
    int64_t Take(hw_spider_metric_block* dst, uint64_t cap, uint64_t* offsets)
    {
        uint64_t total = 0;
        for (const auto& o : out) total += o.size();
        if (total > cap) return -1;
        uint64_t pos = 0;
        for (uint32_t z = 0; z < numZmw; ++z)
        {
            offsets[z] = pos;
            for (const auto& b : out[z]) dst[pos++] = b;
            out[z].clear();
        }
        offsets[numZmw] = pos;
        return (int64_t)pos;
    }
};

}   // namespace

extern "C" {

// literal: keep the reference's two index slips (see above).
void* or_metrics_create(uint32_t numZmw, uint32_t lookback, int32_t enablePrehq, uint32_t zmwStride, int32_t literal)
{
    if (numZmw == 0 || lookback == 0 || zmwStride == 0 || 64 % zmwStride) return nullptr;
    return new MetricSideOracle(numZmw, lookback, enablePrehq != 0, zmwStride, literal != 0);
}

void or_metrics_destroy(void* h) { delete static_cast<MetricSideOracle*>(h); }

// AddMetrics of every ZMW z with z % stride == 0 from one block's HF metrics
// (ceil(numZmw / 64) lanes).
void or_metrics_add(void* h, const hw_basecalling_metrics* lanes) { static_cast<MetricSideOracle*>(h)->Add(lanes); }

// End of a metric block: MarkAsHQ(z) for newly[z] != 0, UpdateLookback,
// GetMetrics.  Returns the blocks written (or -1 when they pass cap: the
// caller retries the GetMetrics with or_metrics_take).
int64_t or_metrics_end_block(void* h, const uint8_t* newly, hw_spider_metric_block* out, uint64_t cap,
                             uint64_t* offsets)
{
    auto* o = static_cast<MetricSideOracle*>(h);
    if (newly)
        for (uint32_t z = 0; z < o->numZmw; ++z)
            if (newly[z]) o->MarkAsHq(z);
    o->UpdateLookback();
    return o->Take(out, cap, offsets);
}

int64_t or_metrics_take(void* h, hw_spider_metric_block* out, uint64_t cap, uint64_t* offsets)
{
    return static_cast<MetricSideOracle*>(h)->Take(out, cap, offsets);
}

// BazAggregator::Flush: MetricBufferManager::Flush then GetMetrics.
int64_t or_metrics_flush(void* h, hw_spider_metric_block* out, uint64_t cap, uint64_t* offsets)
{
    auto* o = static_cast<MetricSideOracle*>(h);
    o->Flush();
    return o->Take(out, cap, offsets);
}

void or_metrics_activity(void* h, uint8_t* out)
{
    auto* o = static_cast<MetricSideOracle*>(h);
    std::copy(o->recentLabel.begin(), o->recentLabel.end(), out);
}

void or_half_bits(const float* x, uint64_t n, uint16_t* out)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = HalfBits(x[i]);
}

void or_half_float(const uint16_t* x, uint64_t n, float* out)
{
    for (uint64_t i = 0; i < n; ++i) out[i] = HalfFloat(x[i]);
}

// One metric block of ZMW z of a lane through the reference's metric types:
// kind 0 ProductionMetrics<uint16_t, half>, 1 CompleteMetrics<uint16_t,
// half>, 2 ProductionMetrics<uint32_t, float>, 3 CompleteMetrics<uint32_t,
// float>, converted.
void or_metric_block_convert(const hw_basecalling_metrics* lane, int32_t z, int32_t kind, hw_spider_metric_block* out)
{
    *out = EmptySpider();
    switch (kind)
    {
    case 0: ProdBlock<uint16_t, Half>(*lane, z).Convert(*out); break;
    case 1: CompleteBlock<uint16_t, Half>(*lane, z).Convert(*out); break;
    case 2: ProdBlock<uint32_t, float>(*lane, z).Convert(*out); break;
    default: CompleteBlock<uint32_t, float>(*lane, z).Convert(*out); break;
    }
}

// Aggregation sequences of the reference's known-answer tests
// (basecaller/dataTypes/test/TestMetrics.cpp:60-146) on ZMWs z0, z1 of a lane.
// test 0 (Production): ProductionMetrics<uint32_t, float>{z0} aggregating
// {z1}; test 1 (Production, half): an empty ProductionMetrics<uint32_t,
// float> aggregating ProductionMetrics<uint16_t, half>{z0} `reps` times;
// test 2 (Aggregate): an empty ProductionMetrics<uint32_t, float> aggregating
// ProductionMetrics<uint16_t, float> {z0} then {z1}; test 3 (Complete):
// CompleteMetrics<uint32_t, float>{z0} aggregating {z1}.  The result is
// converted, and its uncapped counts and aggregate fields are returned in
// raw[0..]: numFrames, pulseWidth, baseWidth, numPulses, numBases,
// numBaselineFrames, numPkmidFrames[0], baselineMean, baselineVar, pkmid[0],
// pkmid[3]; complete: numSandwiches, numHalfSandwiches,
// numPulseLabelStutters, pulseDetectionScore, traceAutoCorrelation,
// pkmax[0], numPkmidBases[0], pkzvar[0], bpzvar[0].
void or_metrics_kat(const hw_basecalling_metrics* lane, int32_t test, int32_t z0, int32_t z1, int32_t reps,
                    hw_spider_metric_block* out, double* raw)
{
    *out = EmptySpider();
    auto prodRaw = [&](const ProdBlock<uint32_t, float>& p) {
        const double v[] = {(double)p.numFrames, (double)p.pulseWidth, (double)p.baseWidth, (double)p.numPulses,
                            (double)p.numBases, (double)p.numBaselineFrames, (double)p.numPkmidFrames[0],
                            (double)p.baselineMean, (double)p.baselineVar, (double)p.pkmid[0], (double)p.pkmid[3]};
        std::copy(v, v + 11, raw);
    };
    if (test == 0)
    {
        ProdBlock<uint32_t, float> m1(*lane, z0), m2(*lane, z1);
        m1.Aggregate(m2);
        m1.Convert(*out);
        prodRaw(m1);
    }
    else if (test == 1)
    {
        ProdBlock<uint16_t, Half> m3(*lane, z0);
        ProdBlock<uint32_t, float> m4;
        for (int i = 0; i < reps; ++i) m4.Aggregate(m3);
        m4.Convert(*out);
        prodRaw(m4);
    }
    else if (test == 2)
    {
        ProdBlock<uint32_t, float> b1;
        ProdBlock<uint16_t, float> b2(*lane, z0), b3(*lane, z1);
        b1.Aggregate(b2);
        b1.Aggregate(b3);
        b1.Convert(*out);
        prodRaw(b1);
    }
    else
    {
        CompleteBlock<uint32_t, float> c1(*lane, z0), c2(*lane, z1);
        c1.Aggregate(c2);
        c1.Convert(*out);
        prodRaw(c1.prod);
        const double v[] = {(double)c1.numSandwiches, (double)c1.numHalfSandwiches, (double)c1.numPulseLabelStutters,
                            (double)c1.pulseDetectionScore, (double)c1.traceAutoCorrelation, (double)c1.pkmax[0],
                            (double)c1.numPkmidBases[0], (double)c1.pkzvar[0], (double)c1.bpzvar[0]};
        std::copy(v, v + 9, raw + 11);
    }
}

}   // extern "C"
