// Per-frame pulse accumulation of one ZMW, shared by the pulse kernel and the
// fused labeler + pulse kernel.
//
// Restates TA/HostPulseAccumulator.{h:64-173, cpp:50-127},
// TA/SubframeLabelManager.h:47-102, DT/Pulse.h:48-237 and the bounded
// per-ZMW pulse vector of DT/BatchVectors.h:105-119
// (TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes).
#pragma once

#include "hw_device.cuh"

namespace hwk {

__device__ __forceinline__ uint16_t ToFixed(float v) { return static_cast<uint16_t>(add_rn(v / .1f, 0.5f)); }

// The open segment (LabelsSegment) and the chunk's outputs of one ZMW.
struct PulseSeg
{
    uint32_t start;
    int16_t first, last, mx, label;
    float total, m2;
    uint32_t n, over;
    float b0, b1, b2;       // StatAccumulator of baseline frames (offset 0)
    float minMean;
    hw_pulse* out;
    // a closed pulse not yet converted (LabelsSegment fields at its end)
    bool pend;
    uint32_t pStart;
    int pWidth;
    float pNum, pTotal, pM2;       // (total + last) + first, total, m2
    int16_t pMx, pLabel;

    __device__ __forceinline__ void Load(const PulseArgs& A, int g, float minMeanIn, hw_pulse* outIn)
    {
        start = A.segStart[g];
        first = A.segFirst[g]; last = A.segLast[g]; mx = A.segMax[g]; label = A.segLabel[g];
        total = A.segTotal[g]; m2 = A.segM2[g];
        n = 0; over = 0;
        b0 = 0.0f; b1 = 0.0f; b2 = 0.0f;
        minMean = minMeanIn;
        out = outIn;
        pend = false;
    }

    // LabelsSegment::ToPulse (HostPulseAccumulator.h:106-138) of the pending
    // pulse, appended to the ZMW's bounded pulse vector.
    __device__ __forceinline__ void Emit(const KParams& k)
    {
        constexpr float maxSignal = 65535 * .1f;
        constexpr float minSignal = 0.0f;
        const int width = pWidth;
        const float rawMean = pNum / (float)width;
        const float rawMid = pTotal / (float)(width - 2);
        const bool keep = ((float)width >= k.widthThresh) || (mul_rn(rawMean, (float)width) >= mul_rn(k.ampThresh, minMean));
        hw_pulse p;
        p.start = pStart;
        p.width = (uint16_t)width;
        p.mean_signal = ToFixed(fmin_std(maxSignal, fmax_std(minSignal, rawMean)));
        p.mid_signal = ToFixed(width < 3 ? 0.0f : fmin_std(maxSignal, fmax_std(minSignal, rawMid)));
        p.max_signal = ToFixed(fmin_std(maxSignal, fmax_std(minSignal, (float)pMx)));
        p.signal_m2 = pM2;
        int lbl = pLabel;
        if (lbl > 2 * kAnalogs) lbl -= 2 * kAnalogs;
        if ((lbl > kAnalogs) & (lbl <= 2 * kAnalogs)) lbl -= kAnalogs;
        p.label = k.analogMap[lbl - 1];
        p.is_reject = keep ? 0 : 1;
        p.pad_[0] = 0; p.pad_[1] = 0;
        if (n < (uint32_t)k.maxCalls) out[n++] = p;
        else ++over;
    }

    // Converts the pending pulse, if any: called after each frame batch and
    // before Store.
    __device__ __forceinline__ void Flush(const KParams& k)
    {
        if (pend)
        {
            Emit(k);
            pend = false;
        }
    }

    __device__ __forceinline__ void Frame(const KParams& k, uint32_t absF, int16_t lb, int16_t signal)
    {
        const bool isUp = (lb > kAnalogs) & (lb <= 2 * kAnalogs);
        const bool boundary = isUp | ((lb == 0) & (label != 0));
        const bool pulseM = label != 0;
        if (boundary & pulseM)
        {
            // The pulse's raw sums wait in the pending slot; ToPulse runs at
            // the end of the frame batch, once for the whole warp, instead of
            // at every frame where some lane of the warp closes a pulse.
            if (pend) Emit(k);
            pend = true;
            pStart = start;
            pWidth = (int)(absF - start);
            pNum = add_rn(add_rn(total, (float)last), (float)first);
            pTotal = total;
            pM2 = m2;
            pMx = mx;
            pLabel = label;
        }
        if (boundary)
        {
            start = absF; first = signal; last = 0; mx = signal; total = 0.0f; m2 = 0.0f; label = lb;
        }
        else
        {
            total = add_rn(total, (float)last);
            m2 = add_rn(m2, mul_rn((float)last, (float)last));
            last = signal;
            mx = signal > mx ? signal : mx;
        }
        if ((!pulseM) & (!boundary))
        {
            const float x = (float)signal;
            b0 += 1.0f; b1 = add_rn(b1, x); b2 = add_rn(b2, mul_rn(x, x));
        }
    }

    __device__ __forceinline__ void Store(const PulseArgs& A, int g, int l, int z, uint32_t* lensOut,
                                          uint32_t* ovfOut, int go) const
    {
        A.segStart[g] = start; A.segFirst[g] = first; A.segLast[g] = last; A.segMax[g] = mx;
        A.segTotal[g] = total; A.segM2[g] = m2; A.segLabel[g] = label;
        lensOut[go] = n;
        ovfOut[go] = over;
        A.bls[l].offset[z] = 0.0f;
        A.bls[l].moment0[z] = b0;
        A.bls[l].moment1[z] = b1;
        A.bls[l].moment2[z] = b2;
    }
};

}   // namespace hwk
