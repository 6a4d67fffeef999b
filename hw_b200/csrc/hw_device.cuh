// Device-side helpers shared by the hw_b200 kernels.
#pragma once

#include <cstring>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <nvtx3/nvToolsExt.h>
#include <stdint.h>

#include "../../include/hw_b200.h"
#include "hw_math.h"
#include "hw_params.h"

namespace hwk {

using namespace hwm;

constexpr int kLane = HW_LANE_SIZE;
constexpr int kAnalogs = HW_NUM_ANALOGS;
constexpr int kBins = HW_NUM_BINS;
constexpr int kStates = HW_NUM_STATES;
constexpr int kLatent = hwp::kLatentFrames;
constexpr int kLookback = hwp::kViterbiStitchLookback;
constexpr int kStitch = hwp::kRoiStitchFrames;

__device__ __forceinline__ float h2f(uint16_t b) { return __half2float(__ushort_as_half(b)); }
__device__ __forceinline__ uint16_t f2h(float f) { return __half_as_ushort(__float2half_rn(f)); }

// ---- Packed pairs (sm_100 f32x2 arithmetic) --------------------------------
// add.rn / mul.rn / fma.rn .f32x2 round each component exactly as the scalar
// .rn instruction does, so a pair of independent scalar chains can be
// evaluated as one packed chain with identical bits and half the issued
// floating-point instructions.  One caution, measured: the code generator
// fuses a packed multiply and a packed add that consumes it into one packed
// fma (one rounding instead of two) even with the explicit .rn and the
// build's -fmad=false, which only holds for scalar arithmetic.  A product
// that feeds an addition is therefore written mulz2(a, b, nz) = fma2(a, b,
// nz) with nz = (-0, -0) read at run time (KParams::negZero): a * b + (-0)
// rounds exactly as a * b (also for a zero product), and an fma is not fused
// with a following add.
__device__ __forceinline__ float2 f2(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "add.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mul.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c)
{
    float2 r;
    asm("{\n\t.reg .b64 pa, pb, pc, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
        "mov.b64 pc, {%6, %7};\n\tfma.rn.f32x2 pr, pa, pb, pc;\n\tmov.b64 {%0, %1}, pr;\n\t}"
        : "=f"(r.x), "=f"(r.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return r;
}
// a * b with the rounding of mul.rn, for products that feed an addition
// (see above); nz holds (-0, -0) from a run-time value.
__device__ __forceinline__ float2 mulz2(float2 a, float2 b, float2 nz) { return fma2(a, b, nz); }

// hw_expf (hw_math.h) of both components: the special-case selects and the
// integer scaling per component, the reduction and the polynomial packed
// (each multiply there feeds an fma, never a packed add).
__device__ __forceinline__ float2 hw_expf2(float2 x, float2 nz)
{
    const bool nanX = x.x != x.x, hiX = x.x > 88.72283935546875f, loX = x.x < -103.97208404541016f;
    const bool nanY = x.y != x.y, hiY = x.y > 88.72283935546875f, loY = x.y < -103.97208404541016f;
    const float2 xc = f2((nanX | hiX | loX) ? 0.0f : x.x, (nanY | hiY | loY) ? 0.0f : x.y);
    const float2 zf = fma2(xc, f2(1.44269504088896341f), f2(0.5f));
    const float2 z = f2(floorf(zf.x), floorf(zf.y));
    float2 r = fma2(z, f2(-0.693359375f), xc);
    r = fma2(z, f2(2.12194440e-4f), r);
    float2 p = fma2(f2(1.9875691500e-4f), r, f2(1.3981999507e-3f));
    p = fma2(p, r, f2(8.3334519073e-3f));
    p = fma2(p, r, f2(4.1665795894e-2f));
    p = fma2(p, r, f2(1.6666665459e-1f));
    p = fma2(p, r, f2(5.0000001201e-1f));
    const float2 r2 = mul2(r, r);
    const float2 y = add2(fma2(p, r2, r), f2(1.0f));
    const int nx = (int)z.x, ny = (int)z.y;
    const int nx1 = nx >> 1, ny1 = ny >> 1;
    float2 out = mulz2(mul2(y, f2(pow2i(nx1), pow2i(ny1))), f2(pow2i(nx - nx1), pow2i(ny - ny1)), nz);
    out.x = loX ? 0.0f : out.x;
    out.y = loY ? 0.0f : out.y;
    out.x = hiX ? __int_as_float(0x7f800000) : out.x;
    out.y = hiY ? __int_as_float(0x7f800000) : out.y;
    out.x = nanX ? x.x : out.x;
    out.y = nanY ? x.y : out.y;
    return out;
}

// hw_expf / hw_expf2 for arguments that are never above 0 (or NaN): the
// E-step's exponents t - tmax and t - llb, where llb >= tmax >= t.  The
// overflow selection of the general routine can never fire there, so it is
// left out; every other step, and so every result, is the same.
__device__ __forceinline__ float hw_expf_np(float x)
{
    const bool isNan = x != x;
    const bool lo = x < -103.97208404541016f;
    const float xc = (isNan | lo) ? 0.0f : x;
    const float z = floorf(fma_rn(xc, 1.44269504088896341f, 0.5f));
    float r = fma_rn(z, -0.693359375f, xc);
    r = fma_rn(z, 2.12194440e-4f, r);
    float p = 1.9875691500e-4f;
    p = fma_rn(p, r, 1.3981999507e-3f);
    p = fma_rn(p, r, 8.3334519073e-3f);
    p = fma_rn(p, r, 4.1665795894e-2f);
    p = fma_rn(p, r, 1.6666665459e-1f);
    p = fma_rn(p, r, 5.0000001201e-1f);
    const float r2 = mul_rn(r, r);
    const float y = add_rn(fma_rn(p, r2, r), 1.0f);
    float out = scale2(y, (int)z);
    out = lo ? 0.0f : out;
    return isNan ? x : out;
}

__device__ __forceinline__ float2 hw_expf2_np(float2 x, float2 nz)
{
    const bool nanX = x.x != x.x, loX = x.x < -103.97208404541016f;
    const bool nanY = x.y != x.y, loY = x.y < -103.97208404541016f;
    const float2 xc = f2((nanX | loX) ? 0.0f : x.x, (nanY | loY) ? 0.0f : x.y);
    const float2 zf = fma2(xc, f2(1.44269504088896341f), f2(0.5f));
    const float2 z = f2(floorf(zf.x), floorf(zf.y));
    float2 r = fma2(z, f2(-0.693359375f), xc);
    r = fma2(z, f2(2.12194440e-4f), r);
    float2 p = fma2(f2(1.9875691500e-4f), r, f2(1.3981999507e-3f));
    p = fma2(p, r, f2(8.3334519073e-3f));
    p = fma2(p, r, f2(4.1665795894e-2f));
    p = fma2(p, r, f2(1.6666665459e-1f));
    p = fma2(p, r, f2(5.0000001201e-1f));
    const float2 r2 = mul2(r, r);
    const float2 y = add2(fma2(p, r2, r), f2(1.0f));
    const int nx = (int)z.x, ny = (int)z.y;
    const int nx1 = nx >> 1, ny1 = ny >> 1;
    float2 out = mulz2(mul2(y, f2(pow2i(nx1), pow2i(ny1))), f2(pow2i(nx - nx1), pow2i(ny - ny1)), nz);
    out.x = loX ? 0.0f : out.x;
    out.y = loY ? 0.0f : out.y;
    out.x = nanX ? x.x : out.x;
    out.y = nanY ? x.y : out.y;
    return out;
}

// Device error word shared by the kernels of one launch: the first failing
// check stores its code; the host reads it after the launch.
struct ErrWord
{
    int* p;
    __device__ void Set(int code) const { if (p) atomicCAS(p, 0, code); }
};

// Per-run constants copied from hwp::Derived into kernel parameter space.
struct KParams
{
    // baseliner
    float cMeanBias, cSigmaBias, meanEmaAlpha, sigmaEmaAlpha, jumpTolCoeff, scaler;
    int pedestal;
    // histogram
    float binSizeMin, binSizeCoeff, fallbackSigma;
    float minFrameCount;
    // dme
    float blVarMin, blVarMax, blVarNominal, logTwoPi, minPulseMean, rpaSum2, rpaMin;
    float shotVarCoeff, refSnr;
    float relAmp[kAnalogs], cv2[kAnalogs];
    float scaleSnrConfTol, pulseAmpReg, snrDropThresh, successConfThresh;
    float snrThresh0, snrThresh1, amft0, amft1;
    float halfLife0, halfLife1;
    int emIterLimit, iterToLimit, updateMethod;
    // labeler
    float trans[kStates][kStates];
    float sqrtHalfPi, sqrt2, sqrt3, roiUpper, roiLower;
    float rcpSqrt2, rcpSqrt3;    // RN(1 / sqrt2), RN(1 / sqrt3)
    // pulses
    float ampThresh, widthThresh;
    int maxCalls;
    uint8_t analogMap[kAnalogs];
    // -0.0f, read at run time by the packed products (mulz2)
    float negZero;
    // labeler, 9-way rows 0, 5, 6, 7, 8 (index 0..4): the transition
    // constants (T[R][5], T[R][9]) of the source groups 5..8 and 9..12, and
    // whether every such row's constants are equal within each group (then
    // the rows take the grouped arg-max)
    float2 grp9[5];
    int grouped9;
};

inline void FillParams(const hw_config& cfg, const hwp::Derived& d, KParams* k)
{
    k->cMeanBias = d.cMeanBias; k->cSigmaBias = d.cSigmaBias;
    k->meanEmaAlpha = d.meanEmaAlpha; k->sigmaEmaAlpha = d.sigmaEmaAlpha;
    k->jumpTolCoeff = d.jumpTolCoeff; k->scaler = d.scaler; k->pedestal = d.pedestal;
    k->binSizeMin = d.binSizeMin; k->binSizeCoeff = cfg.bin_size_coeff;
    k->fallbackSigma = cfg.fallback_baseline_sigma;
    k->minFrameCount = (float)cfg.baseline_stat_min_frame_count;
    k->blVarMin = d.blVarMin; k->blVarMax = d.blVarMax; k->blVarNominal = d.blVarNominal;
    k->logTwoPi = d.logTwoPi; k->minPulseMean = d.minPulseMean; k->rpaSum2 = d.rpaSum2; k->rpaMin = d.rpaMin;
    k->shotVarCoeff = cfg.shot_var_coeff; k->refSnr = cfg.ref_snr;
    for (int a = 0; a < kAnalogs; ++a)
    {
        k->relAmp[a] = cfg.analogs[a].rel_amplitude;
        const float cv = cfg.analogs[a].excess_noise_cv;
        k->cv2[a] = cv * cv;
        k->analogMap[a] = d.analogMap[a];
    }
    k->scaleSnrConfTol = cfg.scale_snr_conf_tol; k->pulseAmpReg = cfg.pulse_amp_regularization;
    k->snrDropThresh = cfg.snr_drop_thresh; k->successConfThresh = cfg.success_confidence_thresh;
    k->snrThresh0 = cfg.min_analog_snr_thresh0; k->snrThresh1 = cfg.min_analog_snr_thresh1;
    k->amft0 = cfg.analog_mix_fraction_threshold[0]; k->amft1 = cfg.analog_mix_fraction_threshold[1];
    k->halfLife0 = cfg.confidence_half_life[0]; k->halfLife1 = cfg.confidence_half_life[1];
    k->emIterLimit = (int)cfg.em_iteration_limit; k->iterToLimit = cfg.iterate_to_limit;
    k->updateMethod = (int)cfg.model_update_method;
    for (int r = 0; r < kStates; ++r)
        for (int c = 0; c < kStates; ++c) k->trans[r][c] = d.trans[r][c];
    k->sqrtHalfPi = d.sqrtHalfPi; k->sqrt2 = d.sqrt2; k->sqrt3 = d.sqrt3;
    k->rcpSqrt2 = 1.0f / d.sqrt2; k->rcpSqrt3 = 1.0f / d.sqrt3;
    k->roiUpper = cfg.roi_upper_threshold; k->roiLower = cfg.roi_lower_threshold;
    k->ampThresh = d.ampThresh; k->widthThresh = d.widthThresh; k->maxCalls = (int)cfg.max_calls_per_zmw;
    k->negZero = -0.0f;
    // Grouped 9-way rows: bitwise-equal, non-NaN constants within each group.
    const int rows9[5] = {0, 5, 6, 7, 8};
    bool grouped = true;
    for (int i = 0; i < 5; ++i)
    {
        const float* t = d.trans[rows9[i]];
        k->grp9[i] = make_float2(t[5], t[9]);
        for (int g = 5; g <= 9; g += 4)
            for (int s = g; s < g + 4; ++s)
                grouped &= (t[s] == t[s]) && std::memcmp(&t[s], &t[g], sizeof(float)) == 0;
        grouped &= (t[0] == t[0]);
    }
    k->grouped9 = grouped ? 1 : 0;
}

// ModelSignalCovar, DetectionModelHost.cpp:237-245
__device__ __forceinline__ float SignalCovar(const KParams& k, float cv2, float mean, float blVar)
{
    float r = blVar;
    r += k.shotVarCoeff * mean;
    r += cv2 * (mean * mean);
    return r;
}

// ---- lane lists (multi-pool launches) ----------------------------------------
// A fused engine keeps the state of all its pools packed lane after lane and
// runs each stage as one launch over a list of its lanes.  Per pool and
// chunk step it publishes a PoolStep (the caller's buffers, the first frame
// and the DME frame-interval centers).

struct PoolStep
{
    const int16_t* trace;       // [lanes][F][64] int16 chunk, or null
    const uint8_t* trace8;      // [lanes][F][64] uint8 chunk, or null
    hw_pulse* pulses;           // [lanes][64][cap]
    uint32_t* lens;             // [lanes][64]
    uint32_t* ovf;              // [lanes][64]
    int32_t firstFrame;         // of the trace chunk
    int32_t F;
    int32_t lane0;              // first engine lane of the pool
    int32_t tModel, tEst;       // DME frame-interval centers
    int32_t hfFlags;            // HF metrics step: kHfReset | kHfFinalize | kHfEmpty
    hw_basecalling_metrics* metrics;   // the pool's HF metrics records [lanes]
};

constexpr int kHfReset = 1, kHfFinalize = 2, kHfEmpty = 4;

struct LaneMap
{
    const int32_t* list = nullptr;     // launch lane -> engine lane; null: single-pool launch
    int n = 0;                         // launch lanes when list is set
    const int32_t* poolOf = nullptr;   // engine lane -> pool
    const uint64_t* frameOff = nullptr;// engine lane -> element offset of its [F][64] block
    const PoolStep* pools = nullptr;   // per pool, this chunk step

    __host__ __device__ bool On() const { return list != nullptr; }
    // launch lanes of a launch over `lanes` lanes
    __host__ __device__ int Lanes(int lanes) const { return list ? n : lanes; }
    __device__ __forceinline__ int Lane(int li) const { return list ? list[li] : li; }
    __device__ __forceinline__ const PoolStep& Pool(int lane) const { return pools[poolOf[lane]]; }
    // element offset of lane's [F][64] block in a per-chunk buffer
    __device__ __forceinline__ size_t Block(int lane, int F) const
    {
        return list ? (size_t)frameOff[lane] : (size_t)lane * F * HW_LANE_SIZE;
    }
    // element offset of lane's [F + extra][64] block (extra frames per lane)
    __device__ __forceinline__ size_t BlockX(int lane, int F, int extra) const
    {
        return list ? (size_t)frameOff[lane] + (size_t)lane * extra * HW_LANE_SIZE
                    : (size_t)lane * (F + extra) * HW_LANE_SIZE;
    }
};

// Thread -> (lane, ZMW) of a launch with one thread per ZMW; false past the
// last launch lane.
__device__ __forceinline__ bool ZmwOf(const LaneMap& m, int lanes, int& l, int& z)
{
    const int gl = blockIdx.x * blockDim.x + threadIdx.x;
    if (gl >= m.Lanes(lanes) * kLane) return false;
    z = gl % kLane;
    l = m.Lane(gl / kLane);
    return true;
}

// ---- kernel argument blocks and launchers ----------------------------------

struct BaselinerArgs
{
    const int16_t* trace;        // [lanes][F][64] (int16 encoding)
    int16_t* out;                // [lanes][F][64]
    hw_baseliner_stats* stats;   // [lanes]
    int16_t* st16;               // [NumI16Slots][nZmw]
    float* st32;                 // [3][nZmw]
    int lanes;
    int F;
    // uint8 encoding: [lanes][F][64], used instead of `trace` when not null;
    // each value is widened to int16 first (BlockView::Extract, BatchData.h:160-180)
    const uint8_t* trace8 = nullptr;
    // lane-list launch: input from map.Pool(lane).trace (or .trace8 when u8
    // is set), `out` and the state packed over the engine's lanes (`lanes` =
    // engine lanes)
    LaneMap map{};
    int u8 = 0;
};

struct DmeArgs
{
    const hw_lane_histogram* hist;
    const hw_baseliner_stats* stats;
    hw_lane_model* models;
    hw_dme_diag* diag;          // may be null
    float* scratch;             // [lanes][3][kBins + 1][64]
    int* err;
    int lanes;
    int32_t tModel, tEst;       // frame-interval centers (model, histogram)
    // Optional EM start [lanes][15][64] (fractions, means, variances), used
    // per ZMW unless its log-likelihood is below the reference start's.
    const float* proposal = nullptr;
    // lane-list launch: frame-interval centers from map.Pool(lane); scratch
    // indexed by launch lane
    LaneMap map{};
    // Optional per-lane phase clock [lanes][8] (SM cycles, thread 0 of the
    // lane): prelude, start choice, E-steps, M-steps, confidence and blend,
    // lane iterations, whole lane, ZMWs that kept the reference start.
    long long* phases = nullptr;
};

struct LabelerArgs
{
    const int16_t* trace;         // [lanes][F][64]
    const hw_lane_model* models;  // [lanes] new models
    int16_t* labels;              // [lanes][F][64]
    int16_t* latOut;              // [lanes][24][64] or null
    float* score;                 // [lanes][64] or null
    // state
    hw_lane_model* latModel;      // [lanes]
    int16_t* latLabel;            // [nZmw]
    int16_t* latRoi;              // [nZmw]
    int16_t* latTrc;              // [nZmw]
    int16_t* prevLat;             // [lanes][24][64]
    uint32_t* tb;                 // [lanes][F + 16][64] scratch
    int lanes;
    int F;
    // best-path decision margin of every label, or null; needs `gap`
    float* margin = nullptr;      // [lanes][F][64]
    float* gap = nullptr;         // [lanes][F + 16][13][64] scratch
    // lane-list launch: per-lane chunk lengths from map.Pool(lane).F, F = the
    // launch's largest
    LaneMap map{};
};

struct PulseArgs
{
    const int16_t* labels;        // [lanes][F][64]
    const int16_t* latTrace;      // [lanes][24][64]
    const int16_t* trace;         // [lanes][F][64]
    const hw_lane_model* models;  // [lanes]
    hw_pulse* pulses;             // [lanes][64][cap]
    uint32_t* lens;               // [lanes][64]
    uint32_t* ovf;                // [lanes][64]
    hw_stat_accum_state* bls;     // [lanes]
    // segment state, [nZmw] each
    uint32_t* segStart;
    int16_t* segFirst;
    int16_t* segLast;
    int16_t* segMax;
    float* segTotal;
    float* segM2;
    int16_t* segLabel;
    int lanes;
    int F;
    uint32_t firstFrame;
    // lane-list launch: outputs and first frame from map.Pool(lane)
    LaneMap map{};
};

// HF metrics in the fused engine: per-lane accumulators (HfLaneBytes each)
// and one lane-list launch per step.
struct HfEngineArgs
{
    LaneMap map;
    void* state;                     // [engine lanes] accumulators
    int cap;
    const hw_baseliner_stats* bs;    // [engine lanes]
    const hw_lane_model* models;
    const float* viterbi;            // [engine lanes][64]
    const hw_stat_accum_state* pd;   // [engine lanes]
    int realtime;
    float frameRate;
    const int16_t* left;
    const int16_t* right;
    const int8_t* feature;
    const float* thr;
    const int8_t* value;
    int nodes;
    float hsw0, hsw1, maxHsw;
};
size_t HfLaneBytes();
cudaError_t LaunchHfInit(void* state, int lanes, cudaStream_t s);
cudaError_t LaunchHfMapped(const HfEngineArgs& a, cudaStream_t s);

int BaselinerNumSlots16(int ft);
cudaError_t LaunchBaseliner(int ft, const BaselinerArgs& a, const KParams& k, cudaStream_t s);
cudaError_t LaunchBaselinerInit(int ft, int16_t* st16, float* st32, int lanes, cudaStream_t s);
cudaError_t LaunchAggReset(hw_baseliner_stats* s, int lanes, cudaStream_t st, const LaneMap& map = LaneMap{});
cudaError_t LaunchAggMerge(hw_baseliner_stats* acc, const hw_baseliner_stats* in, int lanes, cudaStream_t st,
                           const LaneMap& map = LaneMap{});
cudaError_t LaunchHistResetStats(hw_lane_histogram* h, const hw_baseliner_stats* s, int lanes, const KParams& k,
                                 int* err, cudaStream_t st, const LaneMap& map = LaneMap{});
cudaError_t LaunchHistResetBounds(hw_lane_histogram* h, const hw_lane_hist_bounds* b, int lanes, int* err,
                                  cudaStream_t st);
cudaError_t LaunchHistAdd(hw_lane_histogram* h, int16_t* prev, uint8_t* bits, const int16_t* traces, int frames,
                          const hw_lane_model* models, int lanes, cudaStream_t st, const LaneMap& map = LaneMap{});
cudaError_t LaunchInitModels(hw_lane_model* m, const hw_baseliner_stats* s, int lanes, const KParams& k,
                             cudaStream_t st, const LaneMap& map = LaneMap{});
// Zeroes the pulse counts and overflow counters of the listed lanes (pools
// that emit nothing this chunk).
cudaError_t LaunchZeroOutputs(const LaneMap& map, cudaStream_t st);
cudaError_t LaunchDmeEstimate(const DmeArgs& a, const KParams& k, cudaStream_t s);
// fusedPulses: run the pulse accumulator in the labeler kernel (lane-list
// launches only); lanesPerCta: 1, 2 or 4 lanes a block (2 for single-pool
// launches).
cudaError_t LaunchLabeler(const LabelerArgs& a, const KParams& k, cudaStream_t s,
                          const PulseArgs* fusedPulses = nullptr, int lanesPerCta = 2);
cudaError_t LaunchPulses(const PulseArgs& a, const KParams& k, cudaStream_t s);
struct GenArgs;
// Records the thread's last error message (capi.cu) and returns code.
int SetLastError(int code, const char* msg);

// A named NVTX range for the life of the object (header-only NVTX3: nothing
// happens unless a profiler is attached).
struct NvtxRange
{
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};
// Configuration checks and derived constants without heap allocation on success.
int PrepareConfigNoAlloc(const hw_config* cfg, hwp::Derived* d, KParams* k);
cudaError_t LaunchGen(const GenArgs& a, cudaStream_t s);

}   // namespace hwk
