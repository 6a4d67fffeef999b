// Pulse accumulator for sm_100a.
//
// Restates TA/HostPulseAccumulator.{h:64-173, cpp:50-127},
// TA/SubframeLabelManager.h:47-102, DT/Pulse.h:48-237 and the bounded
// per-ZMW pulse vector of DT/BatchVectors.h:105-119
// (TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes).
// One thread per ZMW walks the chunk's labels; the open segment is carried
// across chunks in device state.
#include "hw_device.cuh"

namespace hwk {


__device__ __forceinline__ uint16_t ToFixed(float v) { return static_cast<uint16_t>(add_rn(v / .1f, 0.5f)); }

__global__ void __launch_bounds__(128) PulseKernel(PulseArgs A, KParams k)
{
    int l, z;
    if (!ZmwOf(A.map, A.lanes, l, z)) return;
    const int g = l * kLane + z;
    const int cap = k.maxCalls;
    // outputs, chunk length and first frame: the pool's own in a lane-list launch
    const PoolStep* ps = A.map.On() ? &A.map.Pool(l) : nullptr;
    const int F = ps ? ps->F : A.F;
    const uint32_t firstFrame = ps ? (uint32_t)(ps->firstFrame - kLatent) : A.firstFrame;
    const int go = ps ? (l - ps->lane0) * kLane + z : g;     // ZMW index in the output buffers
    uint32_t* lensOut = ps ? ps->lens : A.lens;
    uint32_t* ovfOut = ps ? ps->ovf : A.ovf;
    uint32_t start = A.segStart[g];
    int16_t first = A.segFirst[g], last = A.segLast[g], mx = A.segMax[g], label = A.segLabel[g];
    float total = A.segTotal[g], m2 = A.segM2[g];
    const float minMean = h2f(A.models[l].analogs[kAnalogs - 1].means[z]);
    const float maxSignal = 65535 * .1f;
    const float minSignal = 0.0f;
    uint32_t n = 0, over = 0;
    hw_pulse* out = (ps ? ps->pulses : A.pulses) + (size_t)go * cap;
    float b0 = 0.0f, b1 = 0.0f, b2 = 0.0f;   // StatAccumulator of baseline frames (offset 0)
    const int16_t* lab = A.labels + A.map.Block(l, F) + z;
    const int16_t* lat = A.latTrace + (size_t)l * kLatent * kLane + z;
    const int16_t* tr = A.trace + A.map.Block(l, F) + z;
    constexpr int kB = 8;
    for (int rel0 = 0; rel0 < F; rel0 += kB)
    {
        // Load the next kB labels and signals ahead of use (F % 8 == 0).
        int16_t lbB[kB], sgB[kB];
#pragma unroll
        for (int j = 0; j < kB; ++j)
        {
            const int r = rel0 + j;
            lbB[j] = __ldg(lab + (size_t)r * kLane);
            sgB[j] = (r < kLatent) ? __ldg(lat + (size_t)r * kLane) : __ldg(tr + (size_t)(r - kLatent) * kLane);
        }
#pragma unroll
        for (int j = 0; j < kB; ++j)
        {
        const int rel = rel0 + j;
        const uint32_t absF = (uint32_t)rel + firstFrame;
        const int16_t lb = lbB[j];
        const int16_t signal = sgB[j];
        const bool isUp = (lb > kAnalogs) & (lb <= 2 * kAnalogs);
        const bool boundary = isUp | ((lb == 0) & (label != 0));
        const bool pulseM = label != 0;
        if (boundary & pulseM)
        {
            // LabelsSegment::ToPulse (HostPulseAccumulator.h:106-138)
            const int width = (int)(absF - start);
            const float rawMean = float(add_rn(add_rn(total, (float)last), (float)first)) / (float)width;
            const float rawMid = total / (float)(width - 2);
            const bool keep = ((float)width >= k.widthThresh) || (mul_rn(rawMean, (float)width) >= mul_rn(k.ampThresh, minMean));
            hw_pulse p;
            p.start = start;
            p.width = (uint16_t)width;
            p.mean_signal = ToFixed(fmin_std(maxSignal, fmax_std(minSignal, rawMean)));
            p.mid_signal = ToFixed(width < 3 ? 0.0f : fmin_std(maxSignal, fmax_std(minSignal, rawMid)));
            p.max_signal = ToFixed(fmin_std(maxSignal, fmax_std(minSignal, (float)mx)));
            p.signal_m2 = m2;
            int lbl = label;
            if (lbl > 2 * kAnalogs) lbl -= 2 * kAnalogs;
            if ((lbl > kAnalogs) & (lbl <= 2 * kAnalogs)) lbl -= kAnalogs;
            p.label = k.analogMap[lbl - 1];
            p.is_reject = keep ? 0 : 1;
            p.pad_[0] = 0; p.pad_[1] = 0;
            if (n < (uint32_t)cap) out[n++] = p;
            else ++over;
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
    }
    A.segStart[g] = start; A.segFirst[g] = first; A.segLast[g] = last; A.segMax[g] = mx;
    A.segTotal[g] = total; A.segM2[g] = m2; A.segLabel[g] = label;
    lensOut[go] = n;
    ovfOut[go] = over;
    A.bls[l].offset[z] = 0.0f;
    A.bls[l].moment0[z] = b0;
    A.bls[l].moment1[z] = b1;
    A.bls[l].moment2[z] = b2;
}

cudaError_t LaunchPulses(const PulseArgs& a, const KParams& k, cudaStream_t s)
{
    if (a.F % 8 != 0) return cudaErrorInvalidValue;
    const int threads = 128;
    const int lanes = a.map.Lanes(a.lanes);
    if (lanes == 0) return cudaSuccess;
    const int blocks = (lanes * kLane + threads - 1) / threads;
    PulseKernel<<<blocks, threads, 0, s>>>(a, k);
    return cudaGetLastError();
}

__global__ void ZeroOutputsKernel(LaneMap map)
{
    int l, z;
    if (!ZmwOf(map, 0, l, z)) return;
    const PoolStep& ps = map.Pool(l);
    const int go = (l - ps.lane0) * kLane + z;
    ps.lens[go] = 0;
    ps.ovf[go] = 0;
}

cudaError_t LaunchZeroOutputs(const LaneMap& map, cudaStream_t s)
{
    if (!map.On() || map.n == 0) return cudaSuccess;
    ZeroOutputsKernel<<<(map.n * kLane + 127) / 128, 128, 0, s>>>(map);
    return cudaGetLastError();
}

}   // namespace hwk
