// HF metrics filter for sm_100a (HFMetricsFilter).
//
// Restates TA/HFMetricsFilterHost.cpp:40-121,
// DT/BasecallingMetricsAccumulator.cpp:40-504, DT/TraceAnalysisMetrics.h:48-200,
// CM/StatAccumulator.h:80-252 and CM/AutocorrAccumulator.cpp:42-103
// (TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes,
// CM = src/basecaller/common).
//
// One block of 64 threads per lane, one thread per ZMW; the accumulators of a
// lane live in global memory between chunks (structure of arrays, so each
// warp access is one contiguous row).  The reference's lane-wide all()/any()
// decisions (StatAccumulator::operator+= and Offset, the empty-channel tests of
// FinalizeMetrics) are block votes, so every ZMW takes the branch the SIMD
// code takes for the whole lane.
#include <string>
#include <vector>

#include "hw_device.cuh"

using namespace hwk;

namespace {

constexpr uint8_t kNoneLabel = 5;      // Pulse::NucleotideLabel::NONE
constexpr int kFeatures = 11;          // ActivityLabeler::NUM_FEATURES

// One lane's BasecallingMetricsAccumulator with its TraceAnalysisMetrics.
struct HfLane
{
    uint16_t pulseFrames[kLane], baseFrames[kLane], sandwiches[kLane], halfSandwiches[kLane], stutters[kLane];
    uint8_t activity[kLane];
    float pkMid[kAnalogs][kLane], bpZvar[kAnalogs][kLane], pkZvar[kAnalogs][kLane], pkMax[kAnalogs][kLane];
    float modelVar[kAnalogs][kLane], modelMean[kAnalogs][kLane];
    uint16_t pkMidFrames[kAnalogs][kLane], pkMidBases[kAnalogs][kLane];
    uint16_t basesBy[kAnalogs][kLane], pulsesBy[kAnalogs][kLane];
    uint32_t startFrame[kLane], numFrames[kLane];
    float pdScore[kLane];
    float blOff[kLane], blM0[kLane], blM1[kLane], blM2[kLane];     // baseline StatAccumulator
    hw_autocorr_accum_state corr;                                   // autocorrelation accumulator
    hw_pulse prev[kLane], prevprev[kLane];
};

struct HfCartDev
{
    const int16_t* left;
    const int16_t* right;
    const int8_t* feature;
    const float* thr;
    const int8_t* value;
    int n;
    float hsw0, hsw1, maxHsw;
};

// One lane's inputs of one step.  viterbi / pd may be null: a pulse batch
// with no frame labeler behind it (zero scores, no baseline frames).
struct HfIn
{
    const hw_pulse* pulses;          // [64][cap] of the lane
    const uint32_t* lens;            // [64], or null: no pulses
    int cap;
    const hw_baseliner_stats* bs;
    const hw_lane_model* model;
    const float* viterbi;            // [64] or null
    const hw_stat_accum_state* pd;   // or null
    uint32_t frames;
    int reset, finalize, realtime;
    float frameRate;
    HfCartDev cart;                  // n == 0: no classifier
    hw_basecalling_metrics* out;     // the lane's record
};

struct HfArgs
{
    HfLane* state;
    const hw_pulse* pulses;
    const uint32_t* lens;
    int cap;
    const hw_baseliner_stats* bs;
    const hw_lane_model* models;
    const float* viterbi;
    const hw_stat_accum_state* pd;
    uint32_t frames;
    int reset, finalize, realtime;
    float frameRate;
    HfCartDev cart;
    hw_basecalling_metrics* out;
};

__device__ __forceinline__ float StatMean(float off, float m0, float m1) { return m1 / m0 + off; }

__device__ __forceinline__ float StatVariance(float m0, float m1, float m2)
{
    float var = mul_rn(m1, m1) / m0;
    var = (m2 - var) / (m0 - 1.0f);
    var = fmax_sse(var, 0.0f);
    return (m0 > 1.0f) ? var : __int_as_float(0x7fffffff);
}

// AutocorrAccumulator::Autocorrelation (AutocorrAccumulator.cpp:42-67).
__device__ float Autocorrelation(const hw_autocorr_accum_state& c, int z)
{
    const hw_stat_accum_state& s = c.basic_stats;
    const float nmk = s.moment0[z] - 4.0f;
    const float mu = StatMean(s.offset[z], s.moment0[z], s.moment1[z]) - s.offset[z];
    float m1x2 = mul_rn(2.0f, s.moment1[z]);
    for (int k = 0; k < 4; ++k) m1x2 = m1x2 - add_rn(c.fbuf[k][z], c.bbuf[k][z]);
    float ac = mul_rn(mu, m1x2 - mul_rn(nmk, mu));
    ac = (c.moment2[z] - ac) / mul_rn(nmk - 1.0f, StatVariance(s.moment0[z], s.moment1[z], s.moment2[z]));
    ac = fmin_sse(fmax_sse(ac, -1.0f), 1.0f);
    return ((nmk < 1.0f) | isnan(ac)) ? __int_as_float(0x7fffffff) : ac;
}

__device__ __forceinline__ float MidSignal(const hw_pulse& p)
{
    return p.width < 3 ? __int_as_float(0x7fffffff) : mul_rn((float)p.mid_signal, 0.1f);
}

// One step of one lane (thread z = ZMW z; the whole 64-thread block takes part
// in the votes).
__device__ void HfStep(HfLane& S, const HfIn& A, int z)
{
    const float kNaN = __int_as_float(0x7fffffff);

    // BasecallingMetricsAccumulator::Reset + TraceAnalysisMetrics::Reset (first chunk of a block)
    if (A.reset)
    {
        S.pulseFrames[z] = 0; S.baseFrames[z] = 0; S.sandwiches[z] = 0; S.halfSandwiches[z] = 0; S.stutters[z] = 0;
        hw_pulse none{};
        none.label = kNoneLabel;
        S.prev[z] = none;
        S.prevprev[z] = none;
        S.activity[z] = 0;
        for (int a = 0; a < kAnalogs; ++a)
        {
            S.pkMid[a][z] = 0; S.bpZvar[a][z] = 0; S.pkZvar[a][z] = 0; S.pkMax[a][z] = 0;
            S.pkMidFrames[a][z] = 0; S.pkMidBases[a][z] = 0; S.basesBy[a][z] = 0; S.pulsesBy[a][z] = 0;
        }
        S.blM0[z] = 0; S.blM1[z] = 0; S.blM2[z] = 0;                         // offset kept
        S.corr.basic_stats.moment0[z] = 0; S.corr.basic_stats.moment1[z] = 0; S.corr.basic_stats.moment2[z] = 0;
        S.corr.moment2[z] = 0;
        for (int k = 0; k < 4; ++k) { S.corr.fbuf[k][z] = 0; S.corr.bbuf[k][z] = 0; }
        S.corr.bidx[0][z] = 0; S.corr.bidx[1][z] = 0;
        S.startFrame[z] = S.startFrame[z] + S.numFrames[z];
        S.numFrames[z] = 0;
        S.pdScore[z] = 0.0f;
    }

    // Count (:348-412)
    S.numFrames[z] += A.frames;
    {
        hw_pulse pp = S.prev[z], ppp = S.prevprev[z];
        const hw_pulse* row = A.pulses + (size_t)z * A.cap;
        const uint32_t n = A.lens ? A.lens[z] : 0u;
        for (uint32_t bi = 0; bi < n; ++bi)
        {
            const hw_pulse p = row[bi];
            const int lb = p.label;
            S.pulseFrames[z] = (uint16_t)(S.pulseFrames[z] + p.width);
            S.pulsesBy[lb][z] = (uint16_t)(S.pulsesBy[lb][z] + 1);
            S.pkMax[lb][z] = fmax_std(S.pkMax[lb][z], mul_rn((float)p.max_signal, 0.1f));
            if (pp.label != kNoneLabel)
            {
                if (pp.label == lb) S.stutters[z] = (uint16_t)(S.stutters[z] + 1);
                const bool abutted = p.start == pp.start + pp.width;
                if (abutted && pp.label != lb) S.halfSandwiches[z] = (uint16_t)(S.halfSandwiches[z] + 1);
                if (ppp.label != kNoneLabel)
                {
                    const bool prevAbutted = pp.start == ppp.start + ppp.width;
                    if (prevAbutted && abutted && ppp.label == lb && ppp.label != pp.label)
                        S.sandwiches[z] = (uint16_t)(S.sandwiches[z] + 1);
                }
            }
            if (!p.is_reject)
            {
                S.baseFrames[z] = (uint16_t)(S.baseFrames[z] + p.width);
                S.basesBy[lb][z] = (uint16_t)(S.basesBy[lb][z] + 1);
                const float mid = MidSignal(p);
                if (!isnan(mid))
                {
                    S.pkMidBases[lb][z] = (uint16_t)(S.pkMidBases[lb][z] + 1);
                    const uint16_t midWidth = (uint16_t)(p.width - 2);
                    S.pkMidFrames[lb][z] = (uint16_t)(S.pkMidFrames[lb][z] + midWidth);
                    S.pkMid[lb][z] = add_rn(S.pkMid[lb][z], mul_rn(mid, (float)midWidth));
                    S.bpZvar[lb][z] = add_rn(S.bpZvar[lb][z], mul_rn(mul_rn(mid, mid), (float)midWidth));
                    S.pkZvar[lb][z] = add_rn(S.pkZvar[lb][z], p.width < 3 ? kNaN : p.signal_m2);
                }
            }
            ppp = pp;
            pp = p;
        }
        S.prev[z] = pp;
        S.prevprev[z] = ppp;
    }

    // AddModels (:311-322)
    for (int a = 0; a < kAnalogs; ++a)
    {
        S.modelVar[a][z] = h2f(A.model->analogs[a].vars[z]);
        S.modelMean[a][z] = h2f(A.model->analogs[a].means[z]);
    }

    // AddBatchMetrics (:324-340)
    const hw_baseliner_stats& B = *A.bs;
    {
        // AutocorrAccumulator::Merge of the chunk's baseline-subtracted
        // statistics (AutocorrAccumulator.cpp:71-103); buffer indices as
        // reconstituted from the lane's first ZMW
        hw_autocorr_accum_state& C = S.corr;
        const hw_autocorr_accum_state& T = B.full_autocorr;
        C.basic_stats.moment0[z] += T.basic_stats.moment0[z];
        C.basic_stats.moment1[z] += T.basic_stats.moment1[z];
        C.basic_stats.moment2[z] += T.basic_stats.moment2[z];
        float m2 = C.moment2[z] + T.moment2[z];
        const int tfbi = T.bidx[0][0], tbbi = T.bidx[1][0];
        const int fbi = C.bidx[0][z], bbi = C.bidx[1][z];
        const int n1 = 4 - tfbi;
        for (int k = 0; k < 4 - n1; ++k)
        {
            const int i = (bbi + k) % 4, j = (tbbi + n1 + k) % 4;
            m2 = add_rn(m2, mul_rn(C.bbuf[i][z], T.fbuf[k][z]));
            C.bbuf[i][z] = T.bbuf[j][z];
        }
        const int n2 = 4 - fbi;
        for (int k = 0; k < n2; ++k) C.fbuf[fbi + k][z] = T.fbuf[k][z];
        C.moment2[z] = m2;
        C.bidx[0][z] = (uint8_t)(fbi + n2);
        C.bidx[1][z] = (uint8_t)((bbi + (4 - n1)) % 4);
    }
    S.pdScore[z] = add_rn(S.pdScore[z], A.viterbi ? A.viterbi[z] : 0.0f);
    {
        // pulse-detector baseline statistics shifted by the background mean,
        // then StatAccumulator::operator+= (StatAccumulator.h:144-166)
        float pOff = 0.0f, pM0 = 0.0f, pM1 = 0.0f, pM2 = 0.0f;
        if (A.pd) { pOff = A.pd->offset[z]; pM0 = A.pd->moment0[z]; pM1 = A.pd->moment1[z]; pM2 = A.pd->moment2[z]; }
        const hw_stat_accum_state& bg = B.background_stats;
        pOff = add_rn(pOff, StatMean(bg.offset[z], bg.moment0[z], bg.moment1[z]));
        float off = S.blOff[z], m0 = S.blM0[z], m1 = S.blM1[z], m2 = S.blM2[z];
        if (!__syncthreads_and(pM0 == 0.0f))
        {
            if (__syncthreads_or(isnan(off)))
            {
                if (isnan(off)) { m0 = 0.0f; m1 = 0.0f; m2 = 0.0f; off = 0.0f; }
            }
            const float w = pM0 / (m0 + pM0);
            float offNew = add_rn(mul_rn(1.0f - w, off), mul_rn(w, pOff));
            offNew = isnan(offNew) ? off : offNew;
            // Offset(value) (:234-246) of the other accumulator, then of this one
            if (!__syncthreads_and(offNew == pOff))
            {
                const float m1n = pM1 + mul_rn(pM0, pOff - offNew);
                const float m2n = pM2 + (mul_rn(m1n, m1n) - mul_rn(pM1, pM1)) / pM0;
                pOff = offNew;
                pM1 = m1n;
                pM2 = (pM0 == 0.0f) ? 0.0f : m2n;
            }
            if (!__syncthreads_and(offNew == off))
            {
                const float m1n = m1 + mul_rn(m0, off - offNew);
                const float m2n = m2 + (mul_rn(m1n, m1n) - mul_rn(m1, m1)) / m0;
                off = offNew;
                m1 = m1n;
                m2 = (m0 == 0.0f) ? 0.0f : m2n;
            }
            m0 += pM0; m1 += pM1; m2 += pM2;
        }
        S.blOff[z] = off; S.blM0[z] = m0; S.blM1[z] = m1; S.blM2[z] = m2;
    }

    if (!A.finalize) return;

    // FinalizeMetrics (:414-500)
    const float blVar = StatVariance(S.blM0[z], S.blM1[z], S.blM2[z]);
    for (int a = 0; a < kAnalogs; ++a)
    {
        const bool allZero = __syncthreads_and((int16_t)S.pkMidBases[a][z] == 0);
        const bool allFewBases = __syncthreads_and((float)S.pkMidBases[a][z] < 2.0f);
        const bool allFewFrames = __syncthreads_and((float)S.pkMidFrames[a][z] < 2.0f);
        if (allZero)
        {
            S.pkMid[a][z] = kNaN; S.bpZvar[a][z] = kNaN; S.pkZvar[a][z] = kNaN;
        }
        else if (allFewBases || allFewFrames)
        {
            S.bpZvar[a][z] = kNaN; S.pkZvar[a][z] = kNaN;
        }
        else
        {
            float bp = S.bpZvar[a][z], pk = S.pkZvar[a][z], mid = S.pkMid[a][z];
            const float nf = (float)S.pkMidFrames[a][z];
            const float nb = (float)S.pkMidBases[a][z];
            bp = (bp - mul_rn(mid, mid) / nf) / nf;
            bp = mul_rn(bp, nb) / (nb - 1.0f);
            bp = bp - blVar / (nf / nb);
            pk = (pk - mul_rn(mid, mid) / nf) / (nf - 1.0f);
            pk = pk - add_rn(bp, blVar);
            const float mv = S.modelVar[a][z];
            bool mask = mv < blVar;
            pk = pk / (mv - blVar);
            mask |= pk < 0.0f;
            pk = mask ? 0.0f : pk;
            const float pkm = mid / nf;
            mask = pkm < 0.0f;
            bp = bp / mul_rn(pkm, pkm);
            mask |= bp < 0.0f;
            bp = mask ? kNaN : bp;
            const int16_t nbi = (int16_t)S.pkMidBases[a][z];
            bool m2 = nbi == 0;
            mid = m2 ? kNaN : mid;
            m2 |= nbi < 2;
            m2 |= (int16_t)S.pkMidFrames[a][z] < 2;
            S.pkMid[a][z] = mid;
            S.bpZvar[a][z] = m2 ? kNaN : bp;
            S.pkZvar[a][z] = m2 ? kNaN : pk;
        }
    }
    {
        const float s = S.pdScore[z] / (float)S.numFrames[z];
        S.pdScore[z] = isnan(s) ? 0.0f : s;
    }
    uint16_t nBasesU = 0, nPulsesU = 0;
    for (int a = 0; a < kAnalogs; ++a)
    {
        nBasesU = (uint16_t)(nBasesU + S.basesBy[a][z]);
        nPulsesU = (uint16_t)(nPulsesU + S.pulsesBy[a][z]);
    }
    const float ac = Autocorrelation(S.corr, z);
    if (A.realtime && A.cart.n > 0)
    {
        // LabelBlock (:65-201)
        float f[kFeatures];
        for (int i = 0; i < kFeatures; ++i) f[i] = 0.0f;
        const float stdDev = sqrtf(blVar);
        const float nBases = (float)nBasesU, nPulses = (float)nPulsesU;
        float pw = (float)S.pulseFrames[z] / nPulses;
        pw = isnan(pw) ? 0.0f : pw;
        float pkmid[kAnalogs];
        for (int a = 0; a < kAnalogs; ++a) pkmid[a] = S.pkMid[a][z] / (float)S.pkMidFrames[a][z];
        const float seconds = (float)S.numFrames[z] / A.frameRate;
        f[0] = nPulses / seconds;
        f[1] = (float)S.sandwiches[z] / nPulses;
        f[1] = isnan(f[1]) ? 0.0f : f[1];
        float hswr = (float)S.halfSandwiches[z] / nPulses;
        hswr = isnan(hswr) ? 0.0f : hswr;
        float hswrExp = add_rn(mul_rn(A.cart.hsw0, f[0]), A.cart.hsw1);
        hswrExp = (hswrExp > A.cart.maxHsw) ? A.cart.maxHsw : hswrExp;
        f[2] = hswr - hswrExp;
        f[3] = S.pdScore[z];
        f[4] = pw;
        f[5] = (float)S.stutters[z] / nPulses;
        f[5] = isnan(f[5]) ? 0.0f : f[5];
        float rel[kAnalogs];
        for (int a = 0; a < kAnalogs; ++a) rel[a] = S.modelMean[a][z];
        float maxamp = rel[0];
        for (int a = 1; a < kAnalogs; ++a) maxamp = fmax_sse(rel[a], maxamp);
        for (int a = 0; a < kAnalogs; ++a) rel[a] = rel[a] / maxamp;
        int lowIdx = 0;
        float minamp = rel[0];
        for (int a = 1; a < kAnalogs; ++a)
        {
            lowIdx = (rel[a] < minamp) ? a : lowIdx;
            minamp = fmin_sse(rel[a], minamp);
        }
        for (int a = 0; a < kAnalogs; ++a)
            f[6] = add_rn(f[6], mul_rn(mul_rn(pkmid[a] / stdDev, (float)S.basesBy[a][z]) / nBases, minamp) / rel[a]);
        f[6] = isnan(f[6]) ? 0.0f : f[6];
        for (int a = 0; a < kAnalogs; ++a) f[7] = fmax_sse(f[7], (S.pkMax[a][z] - pkmid[a]) / stdDev);
        f[7] = isnan(f[7]) ? 0.0f : f[7];
        f[8] = ac;
        for (int a = 0; a < kAnalogs; ++a)
        {
            float t = S.bpZvar[a][z];
            f[9] = add_rn(f[9], (isnan(t) | (lowIdx == a)) ? 0.0f : t);
            t = S.pkZvar[a][z];
            f[10] = add_rn(f[10], (isnan(t) | (lowIdx == a)) ? 0.0f : t);
        }
        f[9] = f[9] / 3.0f;
        f[10] = f[10] / 3.0f;
        // tree walk: bounded by the node count (a malformed table stops, not loops)
        int cur = 0;
        for (int step = 0; step < A.cart.n && A.cart.feature[cur] >= 0; ++step)
        {
            const int fi = A.cart.feature[cur];
            const int nxt = (f[fi < kFeatures ? fi : 0] <= A.cart.thr[cur]) ? A.cart.left[cur] : A.cart.right[cur];
            cur = (nxt >= 0 && nxt < A.cart.n) ? nxt : cur;
        }
        S.activity[z] = (uint8_t)A.cart.value[cur];
    }

    // PopulateBasecallingMetrics (:203-247)
    hw_basecalling_metrics& M = *A.out;
    M.activity_label[z] = S.activity[z];
    M.num_pulse_frames[z] = S.pulseFrames[z];
    M.num_base_frames[z] = S.baseFrames[z];
    M.num_sandwiches[z] = S.sandwiches[z];
    M.num_half_sandwiches[z] = S.halfSandwiches[z];
    M.num_pulse_label_stutters[z] = S.stutters[z];
    M.num_bases[z] = nBasesU;
    M.num_pulses[z] = nPulsesU;
    for (int a = 0; a < kAnalogs; ++a)
    {
        M.pk_mid_signal[a][z] = S.pkMid[a][z];
        M.bp_zvar[a][z] = S.bpZvar[a][z];
        M.pk_zvar[a][z] = S.pkZvar[a][z];
        M.pk_max[a][z] = S.pkMax[a][z];
        M.num_pk_mid_frames[a][z] = S.pkMidFrames[a][z];
        M.num_pk_mid_bases_by_analog[a][z] = S.pkMidBases[a][z];
        M.num_bases_by_analog[a][z] = S.basesBy[a][z];
        M.num_pulses_by_analog[a][z] = S.pulsesBy[a][z];
    }
    M.frame_baseline_dws[z] = StatMean(S.blOff[z], S.blM0[z], S.blM1[z]);
    M.frame_baseline_variance_dws[z] = blVar;
    M.num_frames_baseline[z] = (uint16_t)S.blM0[z];
    M.start_frame[z] = S.startFrame[z];
    M.num_frames[z] = (uint16_t)S.numFrames[z];
    M.autocorrelation[z] = isnan(ac) ? 0.0f : ac;
    M.pulse_detection_score[z] = S.pdScore[z];
    M.pixel_checksum[z] = 0;
}

__global__ void __launch_bounds__(kLane) HfStepKernel(HfArgs A)
{
    const int l = blockIdx.x, z = threadIdx.x;
    HfIn in{A.pulses + (size_t)l * kLane * A.cap, A.lens + (size_t)l * kLane, A.cap, A.bs + l, A.models + l,
            A.viterbi + (size_t)l * kLane, A.pd + l, A.frames, A.reset, A.finalize, A.realtime, A.frameRate, A.cart,
            A.out + l};
    HfStep(A.state[l], in, z);
}

// Lane-list form for the fused engine: flags, outputs and the pulse batch of
// each lane's pool come from its PoolStep.
__global__ void __launch_bounds__(kLane) HfMappedKernel(HfEngineArgs A)
{
    const int li = blockIdx.x, z = threadIdx.x;
    if (li >= A.map.n) return;          // the whole block returns together
    const int l = A.map.Lane(li);
    const PoolStep& ps = A.map.Pool(l);
    const int lp = l - ps.lane0;         // lane within the pool
    const bool empty = (ps.hfFlags & kHfEmpty) != 0;
    HfIn in{ps.pulses + (size_t)lp * kLane * A.cap, empty ? nullptr : ps.lens + (size_t)lp * kLane, A.cap, A.bs + l,
            A.models + l, empty ? nullptr : A.viterbi + (size_t)l * kLane, empty ? nullptr : A.pd + l,
            (uint32_t)ps.F, (ps.hfFlags & kHfReset) != 0, (ps.hfFlags & kHfFinalize) != 0, A.realtime, A.frameRate,
            HfCartDev{A.left, A.right, A.feature, A.thr, A.value, A.nodes, A.hsw0, A.hsw1, A.maxHsw},
            ps.metrics + lp};
    HfStep(static_cast<HfLane*>(A.state)[l], in, z);
}

__global__ void HfInitKernel(HfLane* state, int lanes)
{
    const int l = blockIdx.x, z = threadIdx.x;
    if (l >= lanes) return;
    HfLane& S = state[l];
    S.startFrame[z] = 0; S.numFrames[z] = 0; S.pdScore[z] = 0.0f;
    S.blOff[z] = 0.0f; S.blM0[z] = 0.0f; S.blM1[z] = 0.0f; S.blM2[z] = 0.0f;
    S.corr.basic_stats.offset[z] = 0.0f;
}

int Fail(int code, const std::string& msg) { return hwk::SetLastError(code, msg.c_str()); }

}   // namespace

size_t hwk::HfLaneBytes() { return sizeof(HfLane); }

cudaError_t hwk::LaunchHfInit(void* state, int lanes, cudaStream_t s)
{
    if (lanes == 0) return cudaSuccess;
    HfInitKernel<<<lanes, kLane, 0, s>>>(static_cast<HfLane*>(state), lanes);
    return cudaGetLastError();
}

cudaError_t hwk::LaunchHfMapped(const HfEngineArgs& a, cudaStream_t s)
{
    if (a.map.n == 0) return cudaSuccess;
    HfMappedKernel<<<a.map.n, kLane, 0, s>>>(a);
    return cudaGetLastError();
}

struct hw_hfmetrics
{
    uint32_t lanes = 0, block = 4096, framesSeen = 0;
    float frameRate = 100.0f;
    bool realtime = true;
    HfLane* state = nullptr;
    int16_t* left = nullptr;
    int16_t* right = nullptr;
    int8_t* feature = nullptr;
    float* thr = nullptr;
    int8_t* value = nullptr;
    int nodes = 0;
    float hsw[2] = {0, 0}, maxHsw = 0;
    ~hw_hfmetrics()
    {
        cudaFree(state); cudaFree(left); cudaFree(right); cudaFree(feature); cudaFree(thr); cudaFree(value);
    }
};

extern "C" {

int hw_hfmetrics_create(uint32_t lanes, uint32_t frames_per_block, double frame_rate,
                        int32_t realtime_activity_labels, hw_hfmetrics** out)
{
    if (!out || lanes == 0 || frames_per_block == 0 || !(frame_rate > 0))
        return Fail(HW_ERR_INVALID_ARG, "hw_hfmetrics_create: bad argument");
    *out = nullptr;
    auto h = new hw_hfmetrics;
    h->lanes = lanes;
    h->block = frames_per_block;
    h->frameRate = (float)frame_rate;
    h->realtime = realtime_activity_labels != 0;
    cudaError_t e = cudaMalloc((void**)&h->state, sizeof(HfLane) * lanes);
    if (e == cudaSuccess) e = cudaMemset(h->state, 0, sizeof(HfLane) * lanes);
    if (e == cudaSuccess)
    {
        HfInitKernel<<<lanes, kLane>>>(h->state, (int)lanes);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess)
    {
        delete h;
        return Fail(HW_ERR_CUDA, std::string("hw_hfmetrics_create: ") + cudaGetErrorString(e));
    }
    *out = h;
    return HW_OK;
}

int hw_hfmetrics_destroy(hw_hfmetrics* h)
{
    delete h;
    return HW_OK;
}

int hw_hfmetrics_set_cart(hw_hfmetrics* h, const int16_t* children_left, const int16_t* children_right,
                          const int8_t* feature, const float* threshold, const int8_t* value, uint32_t n_nodes,
                          const float hsw_curve[2], float max_acceptable_halfsandwich_rate)
{
    if (!h || !children_left || !children_right || !feature || !threshold || !value || !hsw_curve || n_nodes == 0 ||
        n_nodes > 32767)
        return Fail(HW_ERR_INVALID_ARG, "hw_hfmetrics_set_cart: bad argument");
    for (uint32_t i = 0; i < n_nodes; ++i)
    {
        if (feature[i] >= kFeatures) return Fail(HW_ERR_INVALID_ARG, "hw_hfmetrics_set_cart: feature index out of range");
        if (feature[i] >= 0 && (children_left[i] < 0 || children_left[i] >= (int)n_nodes || children_right[i] < 0 ||
                                children_right[i] >= (int)n_nodes))
            return Fail(HW_ERR_INVALID_ARG, "hw_hfmetrics_set_cart: child index out of range");
    }
    cudaFree(h->left); cudaFree(h->right); cudaFree(h->feature); cudaFree(h->thr); cudaFree(h->value);
    h->left = h->right = nullptr; h->feature = h->value = nullptr; h->thr = nullptr; h->nodes = 0;
    cudaError_t e = cudaMalloc((void**)&h->left, 2 * n_nodes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->right, 2 * n_nodes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->feature, n_nodes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->thr, 4 * n_nodes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&h->value, n_nodes);
    if (e == cudaSuccess) e = cudaMemcpy(h->left, children_left, 2 * n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->right, children_right, 2 * n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->feature, feature, n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->thr, threshold, 4 * n_nodes, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(h->value, value, n_nodes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_hfmetrics_set_cart: ") + cudaGetErrorString(e));
    h->nodes = (int)n_nodes;
    h->hsw[0] = hsw_curve[0];
    h->hsw[1] = hsw_curve[1];
    h->maxHsw = max_acceptable_halfsandwich_rate;
    return HW_OK;
}

int hw_hfmetrics_process(hw_hfmetrics* h, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                         const hw_baseliner_stats* d_baseliner_stats, const hw_lane_model* d_models,
                         const float* d_viterbi_score, const hw_stat_accum_state* d_pd_baseline_stats,
                         int32_t first_frame, uint32_t frames, hw_basecalling_metrics* d_out, int32_t* emitted,
                         void* stream)
{
    if (!h || !d_pulses || !d_lens || !d_baseliner_stats || !d_models || !d_viterbi_score || !d_pd_baseline_stats ||
        !d_out || max_calls == 0 || frames == 0)
        return Fail(HW_ERR_INVALID_ARG, "hw_hfmetrics_process: bad argument");
    // HFMetricsFilterHost::Process (HFMetricsFilterHost.cpp:80-118)
    HfArgs a{};
    a.state = h->state;
    a.pulses = d_pulses;
    a.lens = d_lens;
    a.cap = (int)max_calls;
    a.bs = d_baseliner_stats;
    a.models = d_models;
    a.viterbi = d_viterbi_score;
    a.pd = d_pd_baseline_stats;
    a.frames = frames;
    a.reset = h->framesSeen == 0;
    const uint32_t last = (uint32_t)(first_frame + (int32_t)frames);
    a.finalize = (last % h->block) < frames;
    a.realtime = h->realtime;
    a.frameRate = h->frameRate;
    a.cart = HfCartDev{h->left, h->right, h->feature, h->thr, h->value, h->nodes, h->hsw[0], h->hsw[1], h->maxHsw};
    a.out = d_out;
    HfStepKernel<<<h->lanes, kLane, 0, reinterpret_cast<cudaStream_t>(stream)>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return Fail(HW_ERR_CUDA, std::string("hw_hfmetrics_process: ") + cudaGetErrorString(e));
    h->framesSeen = a.finalize ? 0 : h->framesSeen + frames;
    if (emitted) *emitted = a.finalize ? 1 : 0;
    return HW_OK;
}

}   // extern "C"
