// Synthetic trace generator (the workloads' stand-in for camera data).
//
// Per ZMW: a baseline level plus N(0, sigma^2) noise; pulses from four analogs
// (uniform choice, amplitude CV per pulse); a pulse starts on a baseline frame
// with probability 1/ipd_mean (or a per-ZMW rate) and ends after each pulse
// frame with probability 1/pulse_width_mean, so widths and gaps are
// geometric; pulse frames add shot-noise variance shot_coeff x amplitude.
// Optional per-ZMW lognormal gain, empty ZMWs, baseline random walk, slow
// amplitude decay and a baseline step.  Random numbers come from a
// counter-based hash of (seed, zmw, frame, slot), so a chunk is reproducible
// from its first frame; the only state carried across chunks is the pulse
// phase, its amplitude and the random-walk offset.
#include "hw_device.cuh"

namespace hwk {

__device__ __forceinline__ uint64_t Mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ uint64_t Draw(uint64_t key, uint64_t ctr) { return Mix64(key ^ Mix64(ctr)); }

__device__ __forceinline__ float U24(uint64_t r, int half)
{
    const uint32_t v = half ? (uint32_t)(r >> 40) : (uint32_t)((r >> 8) & 0xFFFFFFu);
    return (float)v * 5.9604644775390625e-08f;
}

// Marsaglia polar method over up to 8 hash draws.
__device__ __forceinline__ float Normal(uint64_t key, uint64_t ctrBase)
{
    for (int a = 0; a < 8; ++a)
    {
        const uint64_t r = Draw(key, ctrBase + a);
        const float u = 2.0f * U24(r, 0) - 1.0f, v = 2.0f * U24(r, 1) - 1.0f;
        const float s = u * u + v * v;
        if (s > 0.0f && s < 1.0f) return u * sqrtf(-2.0f * hw_logf(s) / s);
    }
    return 0.0f;
}

struct GenArgs
{
    hw_gen_params p;
    int16_t* out;          // [lanes][frames][64]
    uint8_t* inPulse;      // [nZmw]
    float* amp;            // [nZmw]
    float* walk;           // [nZmw]
    int lanes;
    int frames;
    int64_t firstFrame;
    uint64_t zmwOffset;
};

__global__ void __launch_bounds__(256) GenKernel(GenArgs A)
{
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= A.lanes * kLane) return;
    const int l = g / kLane, z = g % kLane;
    const hw_gen_params& P = A.p;
    const uint64_t zmw = A.zmwOffset + (uint64_t)g;
    const uint64_t key = Mix64(P.seed ^ Mix64(zmw * 0x2545F4914F6CDD1Dull + 1));
    // Per-ZMW parameters (frame "-1": counters below 32).
    const float gain = (P.gain_sigma > 0.0f) ? hw_expf(P.gain_sigma * Normal(key, 0)) : 1.0f;
    const float ampScale = (P.amp_scale_sigma > 0.0f) ? hw_expf(P.amp_scale_sigma * Normal(key, 8)) : 1.0f;
    const uint64_t rz = Draw(key, 16);
    const bool empty = U24(rz, 0) < P.empty_fraction;
    const bool stepped = U24(rz, 1) < P.step_fraction;
    float startHazard = 1.0f / P.ipd_mean;
    if (P.rate_max > 0.0f)
    {
        const float rate = P.rate_min + (P.rate_max - P.rate_min) * U24(Draw(key, 17), 0);
        const float gap = fmaxf(1.0f / rate - P.pulse_width_mean, 1.0f);
        startHazard = 1.0f / gap;
    }
    const float endHazard = 1.0f / P.pulse_width_mean;
    bool inp = A.inPulse[g] != 0;
    float amp = A.amp[g];
    float walk = A.walk[g];
    int16_t* out = A.out + (size_t)l * A.frames * kLane + z;
    for (int t = 0; t < A.frames; ++t)
    {
        const int64_t f = A.firstFrame + t;
        const uint64_t base = (uint64_t)(f + 1) * 32;
        const uint64_t r0 = Draw(key, base);
        const float u = U24(r0, 0);
        if (inp)
        {
            if (u < endHazard) inp = false;
        }
        else if (!empty && u < startHazard)
        {
            inp = true;
            int a = (int)(U24(r0, 1) * 4.0f);
            a = a > 3 ? 3 : a;
            float decay = 1.0f;
            if (P.decay_frames > 0)
                decay = 1.0f - P.decay_fraction * fminf((float)f / (float)P.decay_frames, 1.0f);
            const float an = Normal(key, base + 1);
            amp = fmaxf(P.amplitudes[a] * gain * ampScale * decay * (1.0f + P.amp_cv * an), 0.0f);
        }
        if (P.walk_sigma > 0.0f) walk += P.walk_sigma * Normal(key, base + 9);
        const float sig = inp ? amp : 0.0f;
        float level = P.baseline_mean + walk + sig;
        if (stepped && P.step_frame >= 0 && f >= P.step_frame) level += P.step_dn;
        const float sd = sqrtf(P.baseline_sigma * P.baseline_sigma + P.shot_coeff * sig);
        const float v = rintf(level + sd * Normal(key, base + 17));
        out[(size_t)t * kLane] = (int16_t)fminf(fmaxf(v, -32768.0f), 32767.0f);
    }
    A.inPulse[g] = inp ? 1 : 0;
    A.amp[g] = amp;
    A.walk[g] = walk;
}

cudaError_t LaunchGen(const GenArgs& a, cudaStream_t s)
{
    const int threads = 256;
    const int blocks = (a.lanes * kLane + threads - 1) / threads;
    GenKernel<<<blocks, threads, 0, s>>>(a);
    return cudaGetLastError();
}

}   // namespace hwk

// ---- C ABI -------------------------------------------------------------------

struct hw_trace_generator
{
    hw_gen_params p;
    uint32_t lanes;
    uint64_t zmwOffset;
    uint8_t* inPulse = nullptr;
    float* amp = nullptr;
    float* walk = nullptr;
};

extern "C" {

int hw_gen_params_default(int workload, hw_gen_params* p)
{
    if (!p) return HW_ERR_INVALID_ARG;
    memset(p, 0, sizeof(*p));
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

int hw_trace_generator_create(const hw_gen_params* p, uint32_t lanes, uint64_t zmw_offset, hw_trace_generator** out)
{
    if (!p || !out || lanes == 0) return HW_ERR_INVALID_ARG;
    auto g = new hw_trace_generator();
    g->p = *p;
    g->lanes = lanes;
    g->zmwOffset = zmw_offset;
    const size_t n = (size_t)lanes * HW_LANE_SIZE;
    if (cudaMalloc(&g->inPulse, n) != cudaSuccess || cudaMalloc(&g->amp, n * 4) != cudaSuccess ||
        cudaMalloc(&g->walk, n * 4) != cudaSuccess)
    {
        cudaFree(g->inPulse); cudaFree(g->amp); cudaFree(g->walk); delete g;
        cudaGetLastError();
        return HW_ERR_OUT_OF_MEMORY;
    }
    cudaMemset(g->inPulse, 0, n);
    cudaMemset(g->amp, 0, n * 4);
    cudaMemset(g->walk, 0, n * 4);
    *out = g;
    return HW_OK;
}

int hw_trace_generator_destroy(hw_trace_generator* g)
{
    if (!g) return HW_OK;
    cudaFree(g->inPulse); cudaFree(g->amp); cudaFree(g->walk);
    delete g;
    return HW_OK;
}

int hw_trace_generator_next(hw_trace_generator* g, int16_t* d_out, int32_t first_frame, uint32_t frames, void* stream)
{
    if (!g || !d_out || frames == 0) return HW_ERR_INVALID_ARG;
    hwk::GenArgs a{g->p, d_out, g->inPulse, g->amp, g->walk, (int)g->lanes, (int)frames, first_frame, g->zmwOffset};
    return hwk::LaunchGen(a, reinterpret_cast<cudaStream_t>(stream)) == cudaSuccess ? HW_OK : HW_ERR_CUDA;
}

}   // extern "C"
