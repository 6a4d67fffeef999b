// Pulse accumulator for sm_100a.
//
// Restates TA/HostPulseAccumulator.{h:64-173, cpp:50-127},
// TA/SubframeLabelManager.h:47-102, DT/Pulse.h:48-237 and the bounded
// per-ZMW pulse vector of DT/BatchVectors.h:105-119
// (TA = src/basecaller/basecaller/traceAnalysis, DT = src/basecaller/dataTypes).
// One thread per ZMW walks the chunk's labels; the open segment is carried
// across chunks in device state.
#include "pulse_seg.cuh"

namespace hwk {

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
    PulseSeg seg;
    seg.Load(A, g, h2f(A.models[l].analogs[kAnalogs - 1].means[z]),
             (ps ? ps->pulses : A.pulses) + (size_t)go * cap);
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
        for (int j = 0; j < kB; ++j) seg.Frame(k, (uint32_t)(rel0 + j) + firstFrame, lbB[j], sgB[j]);
        seg.Flush(k);
    }
    seg.Store(A, g, l, z, ps ? ps->lens : A.lens, ps ? ps->ovf : A.ovf, go);
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
