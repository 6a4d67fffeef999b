// Configuration-time constants of the trace-analysis chain (host only).
//
// These are the values the reference computes once in its static
// Configure() functions; both the CUDA library and the CPU oracle derive
// their per-run constants here so that the kernels and the checker start from
// the same numbers.  Each block cites the reference lines it restates.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>

#include "../../include/hw_b200.h"
#include "hw_math.h"

namespace hwp {

constexpr int kLane = HW_LANE_SIZE;
constexpr int kAnalogs = HW_NUM_ANALOGS;
constexpr int kBins = HW_NUM_BINS;
constexpr int kStates = HW_NUM_STATES;
constexpr int kMaxScales = 3;
constexpr int kViterbiStitchLookback = 16;     // SubframeScorer.h:45
constexpr int kRoiStitchFrames = 6;            // RoiHost.h:77 RoiFilterDefault
constexpr int kRoiLookForward = 2;
constexpr int kRoiLookBack = 1;
constexpr int kLatentFrames = kViterbiStitchLookback + kRoiLookForward + kRoiStitchFrames;  // 24

// BaselinerParams (traceAnalysis/BaselinerParams.{h,cpp}).
struct FilterParams
{
    int nScales = 0;
    int strides[kMaxScales] = {0, 0, 0};
    int widths[kMaxScales] = {0, 0, 0};
    float sigmaBias = 0.0f;
    float meanBias = 0.0f;

    // BaselinerParams.h:45-60
    int LatentSize() const
    {
        size_t cumStride = 1, minSize = 0;
        for (int i = 0; i < nScales; ++i)
        {
            cumStride *= strides[i];
            minSize += widths[i] * cumStride;
        }
        size_t ret = 1;
        while (ret < minSize) ret *= 2;
        return (int)ret;
    }
    // BaselinerParams.h:62-69
    int AggregateStride() const
    {
        int r = 1;
        for (int i = 0; i < nScales; ++i) r *= strides[i];
        return r;
    }
};

// FilterParamsLookup, BaselinerParams.cpp:30-66
inline bool FilterLookup(int type, FilterParams* p)
{
    auto set = [p](int n, const int* s, const int* w, float sb, float mb) {
        p->nScales = n;
        for (int i = 0; i < n; ++i) { p->strides[i] = s[i]; p->widths[i] = w[i]; }
        p->sigmaBias = sb;
        p->meanBias = mb;
    };
    static const int s3[] = {1, 2, 8}, s2[] = {2, 8};
    static const int wML[] = {11, 17, 61}, wMM[] = {9, 17, 31}, wMS[] = {7, 17, 17};
    static const int wTL[] = {11, 61}, wTM[] = {9, 31}, wTS[] = {7, 17};
    switch (type)
    {
    case HW_FILTER_MULTISCALE_LARGE:  set(3, s3, wML, 2.64f, 0.78f); return true;
    case HW_FILTER_MULTISCALE_MEDIUM: set(3, s3, wMM, 2.41f, 0.69f); return true;
    case HW_FILTER_MULTISCALE_SMALL:  set(3, s3, wMS, 2.15f, 0.63f); return true;
    case HW_FILTER_TWOSCALE_LARGE:    set(2, s2, wTL, 2.71f, 0.60f); return true;
    case HW_FILTER_TWOSCALE_MEDIUM:   set(2, s2, wTM, 2.44f, 0.50f); return true;
    case HW_FILTER_TWOSCALE_SMALL:    set(2, s2, wTS, 2.07f, 0.41f); return true;
    default: return false;
    }
}

// One morphological stage of a multi-stage filter: BlockFilterStage(w, s, nf)
// (BlockFilterStage.h:21-32) with its extremum operator.
struct StageSpec
{
    int width;
    int stride;
    int nf;        // operates on the first NumFrames/nf frames of the block
    bool isMax;    // DilateHgw (max) or ErodeHgw (min)
};

// HostMultiScaleBaseliner.h:110-149.  Lower: erode(w0,s0) dilate(w0); then
// erode(wi,si) dilate(wi).  Upper: dilate(w0,s0) erode(w0); then erode(wi,si)
// dilate(wi) (the same order as the lower filter for i >= 1).
inline int StageSpecs(const FilterParams& fp, bool upper, StageSpec* out)
{
    int n = 0;
    out[n++] = StageSpec{fp.widths[0], fp.strides[0], 1, upper};
    out[n++] = StageSpec{fp.widths[0], 1, fp.strides[0], !upper};
    for (int i = 1; i < fp.nScales; ++i)
    {
        out[n++] = StageSpec{fp.widths[i], fp.strides[i], fp.strides[i - 1], false};
        out[n++] = StageSpec{fp.widths[i], 1, fp.strides[i - 1] * fp.strides[i], true};
    }
    return n;
}

// The 13-state sparse pattern, SubframeScorer.h:55-70.  Row r (destination
// state) has a first entry at column first[r] and one contiguous segment of
// columns [segBegin[r], segEnd[r]); entries are visited in that order.
struct SparseRows
{
    int first[kStates];
    int segBegin[kStates];
    int segEnd[kStates];
};

inline SparseRows TransitionPattern()
{
    SparseRows s{};
    for (int r = 0; r < kStates; ++r)
    {
        if (r == 0 || (r >= 5 && r <= 8)) { s.first[r] = 0; s.segBegin[r] = 5; s.segEnd[r] = 13; }
        else if (r >= 1 && r <= 4) { s.first[r] = r; s.segBegin[r] = r + 4; s.segEnd[r] = r + 5; }
        else { s.first[r] = r - 8; s.segBegin[r] = r - 4; s.segEnd[r] = r - 3; }
    }
    return s;
}

// TransitionMatrix ctor, SubframeScorer.cpp:36-223.  out[to][from] holds the
// log-probability of each sparse entry and -inf elsewhere.  Entries of the
// pattern whose probability is not positive keep the value 0 (the matrix is
// zero-filled before the logs are stored, SparseMatrix.h InitMatrix).
inline void TransitionMatrix(const hw_config& cfg, float out[kStates][kStates])
{
    struct A { float ipd, pw, ipdRatio, pwRatio; } an[kAnalogs];
    for (int i = 0; i < kAnalogs; ++i)
        an[i] = A{cfg.analogs[i].ipd_s, cfg.analogs[i].pulse_width_s,
                  cfg.analogs[i].ipd2_slow_step_ratio, cfg.analogs[i].pw2_slow_step_ratio};
    float dataFloat[kStates][kStates];
    for (auto& row : dataFloat) for (auto& v : row) v = 0.0f;

    // SubframeScorer.cpp:58-74 (the first test reads ipd2SlowStepRatio, as in the reference).
    for (int i = 0; i < kAnalogs; ++i)
    {
        constexpr float delta = 0.01f;
        if (std::abs(an[i].ipdRatio - 1.0f) < delta)
            an[i].pwRatio = (an[i].pwRatio < 1.0f) ? 1.0f - delta : 1.0f + delta;
        if (std::abs(an[i].ipdRatio - 1.0f) < delta)
            an[i].ipdRatio = (an[i].ipdRatio < 1.0f) ? 1.0f - delta : 1.0f + delta;
    }
    float meanIpd = 0.0f;
    for (int i = 0; i < kAnalogs; ++i) meanIpd += an[i].ipd;
    meanIpd = meanIpd / kAnalogs;

    const double frameRate = cfg.frame_rate;
    auto lenProbs = [frameRate](float widthSeconds, float ratio, float r[3]) {
        const double widthFrames = frameRate * widthSeconds;
        ratio = std::max(ratio, 1e-6f);
        const double k1 = (1.0f + ratio) / widthFrames;
        const double k2 = (1.0f + 1.0f / ratio) / widthFrames;
        const double dk = k1 - k2;
        const double c1 = 1.0f - std::exp(-k1);
        const double c2 = 1.0f - std::exp(-k2);
        r[0] = (float)(1 - k1 * c2 / k2 / dk + k2 * c1 / k1 / dk);
        r[1] = (float)(k1 * (c2 * c2) / k2 / dk - k2 * (c1 * c1) / k1 / dk);
        r[2] = (float)(k1 * (c2 * c2) * (1 - c2) / k2 / dk - k2 * (c1 * c1) * (1 - c1) / k1 / dk);
    };

    float ipdLen[kAnalogs][3];
    for (int i = 0; i < kAnalogs; ++i) lenProbs(an[i].ipd, an[i].ipdRatio, ipdLen[i]);
    float alpha[kAnalogs];
    for (int i = 0; i < kAnalogs; ++i)
        alpha[i] = cfg.viterbi_alpha * 0.25f * (ipdLen[i][0] + ipdLen[i][1]);
    float alphaSum = 0.0f;
    for (int i = 0; i < kAnalogs; ++i) alphaSum += alpha[i];

    float meanLen[3];
    lenProbs(meanIpd, 0.0f, meanLen);
    const float meanIpd3m = 1 - meanLen[0] - meanLen[1];
    const float pulseStartProb = meanLen[2] / meanIpd3m;
    dataFloat[0][0] = 1.0f - pulseStartProb;
    for (int i = 0; i < kAnalogs; ++i)
    {
        const int full = i + 1, up = i + 1 + kAnalogs, down = i + 1 + 2 * kAnalogs;
        float lp[3];
        lenProbs(an[i].pw, an[i].pwRatio, lp);
        const float gamma = cfg.viterbi_gamma * lp[0] / (1 + alphaSum);
        const float beta = cfg.viterbi_beta * lp[1];
        dataFloat[up][0] = 0.25f * pulseStartProb;
        dataFloat[0][up] = gamma;
        dataFloat[down][up] = beta;
        dataFloat[full][up] = 1 - gamma - gamma * alphaSum - beta;
        const float prob3ms = 1.0f - lp[0] - lp[1];
        dataFloat[down][full] = lp[2] / prob3ms;
        dataFloat[full][full] = 1.0f - dataFloat[down][full];
        dataFloat[0][down] = 1 - alphaSum;
        for (int j = 0; j < kAnalogs; ++j)
        {
            const int upPrime = j + 1 + kAnalogs;
            dataFloat[upPrime][down] = alpha[j];
            dataFloat[upPrime][up] = gamma * alpha[j];
        }
    }

    const SparseRows sp = TransitionPattern();
    const float ninf = -std::numeric_limits<float>::infinity();
    for (int r = 0; r < kStates; ++r)
        for (int c = 0; c < kStates; ++c) out[r][c] = ninf;
    for (int r = 0; r < kStates; ++r)
    {
        out[r][sp.first[r]] = 0.0f;
        for (int c = sp.segBegin[r]; c < sp.segEnd[r]; ++c) out[r][c] = 0.0f;
    }
    for (int r = 0; r < kStates; ++r)
        for (int c = 0; c < kStates; ++c)
            if (dataFloat[r][c] > 0.0f) out[r][c] = std::log(dataFloat[r][c]);
}

// Per-run constants.  Names follow the reference's static members.
struct Derived
{
    FilterParams fp;
    int aggStride;
    // MultiScaleBaseliner::Configure (MultiScaleBaseliner.cpp:53-82) and
    // LaneBaseliner ctor (HostMultiScaleBaseliner.h:64-72)
    float cMeanBias, cSigmaBias, meanEmaAlpha, sigmaEmaAlpha, jumpTolCoeff;
    float scaler;
    int16_t pedestal;
    uint32_t baselinerStartupLatency;
    // TraceHistogramAccumHost (TraceHistogramAccumHost.cpp:96-126)
    float binSizeMin;
    // CoreDMEstimator::Configuration (CoreDMEstimator.h:67-93)
    float blVarNominal, blVarMin, blVarMax;
    float logTwoPi;           // DmeEmHost.cpp:383 std::log(2 pi)
    float minPulseMean;       // DmeEmHost.cpp:520
    float rpaSum2;            // rpa.square().sum() in SSE packet order
    float rpaMin;
    // Frame labeler
    float trans[kStates][kStates];
    float sqrtHalfPi;         // SubframeScorer.h:211
    float sqrt2, sqrt3;       // RoiHost.h:93-95
    // PulseAccumulator::InitFactory (PulseAccumulator.cpp:48-76)
    float ampThresh, widthThresh;
    uint8_t analogMap[kAnalogs];
};

inline int NucleotideIndex(char c)
{
    const char tbl[] = {'A', 'C', 'G', 'T', 'N', '-'};
    for (int i = 0; i < 6; ++i) if (tbl[i] == c) return i;
    return -1;
}

inline bool Derive(const hw_config& cfg, Derived* d, std::string* err)
{
    if (!FilterLookup(cfg.filter_type, &d->fp)) { *err = "unknown baseline filter type"; return false; }
    d->aggStride = d->fp.AggregateStride();
    d->cMeanBias = d->fp.meanBias * std::exp2(cfg.mean_bias_adjust);
    d->cSigmaBias = d->fp.sigmaBias * std::exp2(cfg.sigma_bias_adjust);
    d->meanEmaAlpha = std::pow(0.5f, 1.0f / cfg.mean_ema_scale_strides);
    d->sigmaEmaAlpha = std::exp2(-1.0f / cfg.sigma_ema_scale_strides);
    const float js = cfg.jump_suppression;
    d->jumpTolCoeff = (js > 0.0f) ? 1.0f / js : std::numeric_limits<float>::infinity();
    d->scaler = cfg.photoelectron_sensitivity;
    d->pedestal = cfg.pedestal;
    {
        // MultiScaleBaseliner.h:86-99
        const float meanScale = -1.0f / std::log2(d->meanEmaAlpha);
        const float sigmaScale = -1.0f / std::log2(d->sigmaEmaAlpha);
        const float maxScaleStrides = std::max(meanScale, sigmaScale);
        d->baselinerStartupLatency = (uint32_t)(size_t)((size_t)d->fp.LatentSize()
                                                        + maxScaleStrides * (size_t)d->aggStride);
    }
    d->binSizeMin = cfg.bin_size_low_bound_coeff * std::max(1.0f, cfg.photoelectron_sensitivity);

    const float ss = cfg.photoelectron_sensitivity;
    d->blVarNominal = (2.0f * ss) * (2.0f * ss);
    {
        constexpr float oneTwelfth = 1.0f / 12.0f;
        const float s1 = std::max(ss, 1.0f);
        d->blVarMin = s1 * s1 * oneTwelfth;
        constexpr float headroom = 6.0f * 6.0f;
        d->blVarMax = headroom * d->blVarNominal;
    }
    constexpr float pi_f = 3.1415926536f;
    d->logTwoPi = std::log(2.0f * pi_f);
    d->minPulseMean = std::max(1.0f, ss);
    {
        float q[4];
        for (int a = 0; a < kAnalogs; ++a) q[a] = cfg.analogs[a].rel_amplitude * cfg.analogs[a].rel_amplitude;
        // Eigen SSE predux order for a 4-float packet: (q0 + q2) + (q1 + q3)
        d->rpaSum2 = (q[0] + q[2]) + (q[1] + q[3]);
        float m = cfg.analogs[0].rel_amplitude;
        for (int a = 1; a < kAnalogs; ++a) m = std::min(m, cfg.analogs[a].rel_amplitude);
        d->rpaMin = m;
    }

    TransitionMatrix(cfg, d->trans);
    d->sqrtHalfPi = std::sqrt(0.5f * pi_f);
    d->sqrt2 = std::sqrt(2.0f);
    d->sqrt3 = std::sqrt(3.0f);

    d->widthThresh = cfg.xsp_width_thresh;
    d->ampThresh = static_cast<float>(cfg.xsp_amp_thresh / (1.0 - cfg.xsp_amp_thresh));
    for (int a = 0; a < kAnalogs; ++a)
    {
        const int idx = NucleotideIndex(cfg.analogs[a].base_label);
        if (idx < 0) { *err = "bad analog base label"; return false; }
        d->analogMap[a] = (uint8_t)idx;
    }
    return true;
}

// Reference defaults plus the analog set of the synthetic workloads.
inline void DefaultConfig(hw_config* c)
{
    std::memset(c, 0, sizeof(*c));
    c->frame_rate = 100.0;
    c->photoelectron_sensitivity = 1.0f;
    c->ref_snr = 10.0f;
    c->shot_var_coeff = 0.5f;
    c->pedestal = 0;
    const char labels[4] = {'A', 'C', 'G', 'T'};
    const float relAmp[4] = {4.0f, 2.5f, 1.6f, 1.0f};
    for (int a = 0; a < kAnalogs; ++a)
    {
        c->analogs[a].base_label = labels[a];
        c->analogs[a].rel_amplitude = relAmp[a];
        c->analogs[a].excess_noise_cv = 0.1f;
        c->analogs[a].pulse_width_s = 0.08f;
        c->analogs[a].ipd_s = 0.14f;
        c->analogs[a].pw2_slow_step_ratio = 0.0f;
        c->analogs[a].ipd2_slow_step_ratio = 0.0f;
    }
    c->filter_type = HW_FILTER_MULTISCALE_LARGE;
    c->mean_bias_adjust = 0.0f;
    c->sigma_bias_adjust = 0.0f;
    c->mean_ema_scale_strides = 0.0f;
    c->sigma_ema_scale_strides = 512.0f;
    c->jump_suppression = 0.0f;
    c->bin_size_coeff = 0.2f;
    c->bin_size_low_bound_coeff = 1.0f;
    c->baseline_stat_min_frame_count = 50u;
    c->fallback_baseline_sigma = 10.0f;
    c->num_frames_pre_accum_stats = 1000u;
    c->min_frames_for_estimate = 4000u;
    c->analog_mix_fraction_threshold[0] = 0.039f / 3;
    c->analog_mix_fraction_threshold[1] = 0.039f;
    c->scale_snr_conf_tol = 1.0f;
    c->em_iteration_limit = 20;
    c->gtest_stat_factor = -1.0f;
    c->iterate_to_limit = 0;
    c->min_analog_snr_thresh0 = 2.0f;
    c->min_analog_snr_thresh1 = 4.0f;
    c->pulse_amp_regularization = 0.0f;
    c->model_update_method = 1;
    c->snr_drop_thresh = 1.0f;
    c->success_confidence_thresh = 0.10f;
    c->confidence_half_life[0] = 4096.0f;
    c->confidence_half_life[1] = 12000.0f;
    c->viterbi_alpha = 1.0f;
    c->viterbi_beta = 1.0f;
    c->viterbi_gamma = 1.0f;
    c->roi_filter_type = HW_ROI_DEFAULT;
    c->roi_upper_threshold = 7.0f;
    c->roi_lower_threshold = 2.0f;
    c->max_calls_per_zmw = 48;
    c->xsp_amp_thresh = 0.70;
    c->xsp_width_thresh = 3.5f;
    c->model_estimation_mode = HW_DYNAMIC_ESTIMATIONS;
    c->static_baseline_mean = 0.0f;
    c->static_baseline_variance = 33.0f;     // StaticDetModelConfig.h:44
}

// ValidateConfig<> checks of the reference configs and Configure() asserts.
inline bool Validate(const hw_config& c, std::string* err)
{
    FilterParams fp;
    if (!FilterLookup(c.filter_type, &fp)) { *err = "filter_type out of range"; return false; }
    if (!std::isfinite(c.mean_bias_adjust) || !std::isfinite(c.sigma_bias_adjust))
    { *err = "MeanBiasAdjust/SigmaBiasAdjust must be finite"; return false; }
    if (std::isnan(c.sigma_ema_scale_strides) || std::signbit(c.sigma_ema_scale_strides))
    { *err = "SigmaEmaScaleStrides may not be negative, -0, or NaN"; return false; }
    if (c.mean_ema_scale_strides < 0) { *err = "MeanEmaScaleStrides must be >= 0"; return false; }
    if (c.jump_suppression < 0) { *err = "JumpSuppression must be >= 0"; return false; }
    if (c.bin_size_coeff <= 0.0f) { *err = "BinSizeCoeff must be positive"; return false; }
    if (c.fallback_baseline_sigma <= 0.0f) { *err = "FallBackBaselineSigma must be positive"; return false; }
    if (c.bin_size_low_bound_coeff < 0.0f) { *err = "BinSizeLowBoundCoeff must be non-negative"; return false; }
    const float* amft = c.analog_mix_fraction_threshold;
    if (!(std::isfinite(amft[1]) && amft[1] <= 0.25f)) { *err = "AnalogMixFractionThreshold upper bound"; return false; }
    if (!(std::isfinite(amft[0]) && amft[0] <= amft[1])) { *err = "AnalogMixFractionThreshold lower bound"; return false; }
    if (c.confidence_half_life[0] < 0.0f || c.confidence_half_life[1] < 0.0f)
    { *err = "ConfidenceHalfLife may not be negative"; return false; }
    if (c.model_update_method > 2) { *err = "ModelUpdateMethod must be 0, 1 or 2"; return false; }
    if (c.xsp_width_thresh < 0.0f) { *err = "XspWidthThresh must be non-negative"; return false; }
    if (c.xsp_amp_thresh < 0.0 || c.xsp_amp_thresh > 1.0) { *err = "XspAmpThresh must be in [0, 1]"; return false; }
    if (c.max_calls_per_zmw == 0) { *err = "maxCallsPerZmw must be positive"; return false; }
    if (!(c.photoelectron_sensitivity > 0.0f) || !std::isfinite(c.photoelectron_sensitivity))
    { *err = "photoelectronSensitivity must be finite and positive"; return false; }
    for (int a = 0; a < kAnalogs; ++a)
    {
        if (c.analogs[a].rel_amplitude <= 0.0f)
        { *err = "Bad relative amplitude in analog properties. Relative amplitudes must be greater than zero."; return false; }
        if (NucleotideIndex(c.analogs[a].base_label) < 0) { *err = "bad analog base label"; return false; }
    }
    if (c.roi_filter_type != HW_ROI_DEFAULT && c.roi_filter_type != HW_ROI_NOOP)
    { *err = "roi filter type out of range"; return false; }
    if (c.model_estimation_mode < 0 || c.model_estimation_mode > 2)
    { *err = "model estimation mode out of range"; return false; }
    if (c.model_estimation_mode == HW_FIXED_ESTIMATIONS && !(c.static_baseline_variance >= 0.0f))
    { *err = "StaticDetModelConfig baselineVariance must be non-negative"; return false; }
    return true;
}

// The fixed detection model of FixedModelBatchAnalyzer (analyzer/
// BatchAnalyzer.cpp:119-144) with StaticDetModelConfig::SetupAnalogs
// (dataTypes/configs/StaticDetModelConfig.h:53-68): baseline mean/variance
// from the config, analog a at mean = blMean + relAmp[a] * refSnr * sqrt(blVar)
// and variance blVar + mean + (cv[a] * mean)^2, stored as fp16 in every ZMW.
// Weights and confidence are 0: the labeler and the pulse accumulator read
// only means and variances.
inline void StaticModel(const hw_config& c, hw_lane_model* m)
{
    std::memset(m, 0, sizeof(*m));
    const float blMean = c.static_baseline_mean;
    const float blVar = c.static_baseline_variance;
    const float refSignal = c.ref_snr * std::sqrt(blVar);
    for (int z = 0; z < kLane; ++z)
    {
        m->baseline.means[z] = hwm::f32_to_f16_bits(blMean);
        m->baseline.vars[z] = hwm::f32_to_f16_bits(blVar);
    }
    for (int a = 0; a < kAnalogs; ++a)
    {
        const float mean = blMean + c.analogs[a].rel_amplitude * refSignal;
        const float cm = c.analogs[a].excess_noise_cv * mean;
        const float var = (blVar + mean) + cm * cm;
        for (int z = 0; z < kLane; ++z)
        {
            m->analogs[a].means[z] = hwm::f32_to_f16_bits(mean);
            m->analogs[a].vars[z] = hwm::f32_to_f16_bits(var);
        }
    }
}

}   // namespace hwp
