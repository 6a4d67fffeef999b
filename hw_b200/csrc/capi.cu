// C ABI of hw_b200: per-pool handles that own the device state of each filter
// and launch the sm_100a kernels.  See include/hw_b200.h for the contract.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "hw_device.cuh"


using namespace hwk;

namespace {

thread_local std::string g_lastError = "";

int Fail(int code, const std::string& msg)
{
    g_lastError = msg;
    return code;
}

int CudaFail(cudaError_t e, const char* where)
{
    g_lastError = std::string(where) + ": " + cudaGetErrorString(e);
    return HW_ERR_CUDA;
}

#define HW_CUDA(call, where) do { cudaError_t e_ = (call); if (e_ != cudaSuccess) return CudaFail(e_, where); } while (0)

template <typename T>
int DevAlloc(T** p, size_t count, const char* where)
{
    *p = nullptr;
    if (count == 0) return HW_OK;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess)
    {
        *p = nullptr;
        if (e == cudaErrorMemoryAllocation) { cudaGetLastError(); return Fail(HW_ERR_OUT_OF_MEMORY, std::string(where) + ": out of device memory"); }
        return CudaFail(e, where);
    }
    return HW_OK;
}

int PrepareConfig(const hw_config* cfg, hwp::Derived* d, KParams* k)
{
    if (!cfg) return Fail(HW_ERR_INVALID_ARG, "config is NULL");
    std::string err;
    if (!hwp::Validate(*cfg, &err)) return Fail(HW_ERR_INVALID_ARG, "invalid configuration: " + err);
    if (!hwp::Derive(*cfg, d, &err)) return Fail(HW_ERR_INVALID_ARG, "invalid configuration: " + err);
    if (cfg->gtest_stat_factor >= 0.0f)
        return Fail(HW_ERR_UNSUPPORTED, "GTestStatFactor >= 0 (G-test confidence factor) is not built; the reference default is -1");
    if (cfg->roi_filter_type != HW_ROI_DEFAULT)
        return Fail(HW_ERR_UNSUPPORTED, "RoiFilterNoOp is not built; the reference default is RoiFilterDefault");
    FillParams(*cfg, *d, k);
    return HW_OK;
}

inline cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Reads back and clears a device error word (synchronous).
int TakeDeviceError(int* dErr, cudaStream_t s, const char* where)
{
    int h = 0;
    HW_CUDA(cudaMemcpyAsync(&h, dErr, sizeof(int), cudaMemcpyDeviceToHost, s), where);
    HW_CUDA(cudaStreamSynchronize(s), where);
    if (h != 0)
    {
        HW_CUDA(cudaMemsetAsync(dErr, 0, sizeof(int), s), where);
        return h;
    }
    return HW_OK;
}

}   // namespace

int hwk::SetLastError(int code, const char* msg)
{
    g_lastError = msg;
    return code;
}

int hwk::PrepareConfigNoAlloc(const hw_config* cfg, hwp::Derived* d, KParams* k)
{
    return PrepareConfig(cfg, d, k);
}

// ---------------------------------------------------------------------------

struct hw_baseliner
{
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    uint32_t poolId = 0, lanes = 0, F = 0;
    int slots16 = 0;
    int16_t* st16 = nullptr;
    float* st32 = nullptr;
};

struct hw_blstats_aggregator
{
    uint32_t poolId = 0, lanes = 0;
    hw_baseliner_stats* acc = nullptr;
    hw_frame_interval fi{0, 0};
};

struct hw_histogram
{
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    uint32_t poolId = 0, lanes = 0;
    hw_lane_histogram* hist = nullptr;
    int16_t* edgePrev = nullptr;
    uint8_t* edgeBits = nullptr;
    int* err = nullptr;
    bool initialized = false;
    hw_frame_interval fi{0, 0};
};

struct hw_dme
{
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    uint32_t poolId = 0, lanes = 0;
    float* scratch = nullptr;
    int* err = nullptr;
    long long* phases = nullptr;     // per-lane phase clock when profiling
};

struct hw_labeler
{
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    uint32_t poolId = 0, lanes = 0, F = 0;
    hw_lane_model* latModel = nullptr;
    int16_t* latLabel = nullptr;
    int16_t* latRoi = nullptr;
    int16_t* latTrc = nullptr;
    int16_t* prevLat = nullptr;
    uint32_t* tb = nullptr;
    float* gap = nullptr;     // decision gaps, allocated on the first call that asks for margins
};

struct hw_pulse_accumulator
{
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    uint32_t poolId = 0, lanes = 0, F = 0;
    uint32_t* segStart = nullptr;
    int16_t* segFirst = nullptr;
    int16_t* segLast = nullptr;
    int16_t* segMax = nullptr;
    float* segTotal = nullptr;
    float* segM2 = nullptr;
    int16_t* segLabel = nullptr;
};

extern "C" {

const char* hw_last_error_string(void) { return g_lastError.c_str(); }

const char* hw_version(void) { return "hw_b200 0.1.0 (sm_100a)"; }

int hw_config_default(hw_config* cfg)
{
    if (!cfg) return Fail(HW_ERR_INVALID_ARG, "config is NULL");
    hwp::DefaultConfig(cfg);
    return HW_OK;
}

int hw_config_validate(const hw_config* cfg)
{
    hwp::Derived d;
    KParams k;
    return PrepareConfig(cfg, &d, &k);
}

int hw_transition_matrix(const hw_config* cfg, float out[HW_NUM_STATES][HW_NUM_STATES])
{
    if (!cfg || !out) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    hwp::TransitionMatrix(*cfg, out);
    return HW_OK;
}

uint32_t hw_labeler_latent_frames(void) { return (uint32_t)kLatent; }

// ---- Baseliner -------------------------------------------------------------

int hw_baseliner_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, uint32_t frames_per_chunk,
                        hw_baseliner** out)
{
    if (!out) return Fail(HW_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto b = std::make_unique<hw_baseliner>();
    int rc = PrepareConfig(cfg, &b->d, &b->k);
    if (rc) return rc;
    if (lanes == 0) return Fail(HW_ERR_INVALID_ARG, "lanes must be positive");
    if (frames_per_chunk == 0 || frames_per_chunk % (uint32_t)b->d.aggStride != 0)
        return Fail(HW_ERR_INVALID_ARG, "frames_per_chunk must be a positive multiple of the filter's aggregate stride");
    b->cfg = *cfg;
    b->poolId = pool_id;
    b->lanes = lanes;
    b->F = frames_per_chunk;
    b->slots16 = BaselinerNumSlots16(cfg->filter_type);
    const size_t nZmw = (size_t)lanes * kLane;
    if ((rc = DevAlloc(&b->st16, (size_t)b->slots16 * nZmw, "hw_baseliner_create"))) return rc;
    if ((rc = DevAlloc(&b->st32, 3 * nZmw, "hw_baseliner_create"))) { cudaFree(b->st16); return rc; }
    HW_CUDA(LaunchBaselinerInit(cfg->filter_type, b->st16, b->st32, (int)lanes, 0), "hw_baseliner_create");
    HW_CUDA(cudaDeviceSynchronize(), "hw_baseliner_create");
    *out = b.release();
    return HW_OK;
}

int hw_baseliner_destroy(hw_baseliner* b)
{
    if (!b) return HW_OK;
    cudaFree(b->st16);
    cudaFree(b->st32);
    delete b;
    return HW_OK;
}

int hw_baseliner_startup_latency(const hw_baseliner* b, uint32_t* frames)
{
    if (!b || !frames) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    *frames = b->d.baselinerStartupLatency;
    return HW_OK;
}

int hw_baseliner_process(hw_baseliner* b, const int16_t* d_trace, int32_t first_frame, int16_t* d_out,
                         hw_baseliner_stats* d_stats, void* stream)
{
    (void)first_frame;
    if (!b || !d_trace || !d_out || !d_stats) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    BaselinerArgs a{d_trace, d_out, d_stats, b->st16, b->st32, (int)b->lanes, (int)b->F};
    HW_CUDA(LaunchBaseliner(b->cfg.filter_type, a, b->k, S(stream)), "hw_baseliner_process");
    return HW_OK;
}

int hw_baseliner_process_u8(hw_baseliner* b, const uint8_t* d_trace, int32_t first_frame, int16_t* d_out,
                            hw_baseliner_stats* d_stats, void* stream)
{
    (void)first_frame;
    if (!b || !d_trace || !d_out || !d_stats) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    BaselinerArgs a{nullptr, d_out, d_stats, b->st16, b->st32, (int)b->lanes, (int)b->F, d_trace};
    HW_CUDA(LaunchBaseliner(b->cfg.filter_type, a, b->k, S(stream)), "hw_baseliner_process_u8");
    return HW_OK;
}

// ---- Aggregator --------------------------------------------------------------

int hw_blstats_aggregator_create(uint32_t pool_id, uint32_t lanes, hw_blstats_aggregator** out)
{
    if (!out || lanes == 0) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    *out = nullptr;
    auto a = std::make_unique<hw_blstats_aggregator>();
    a->poolId = pool_id;
    a->lanes = lanes;
    int rc = DevAlloc(&a->acc, lanes, "hw_blstats_aggregator_create");
    if (rc) return rc;
    HW_CUDA(LaunchAggReset(a->acc, (int)lanes, 0), "hw_blstats_aggregator_create");
    HW_CUDA(cudaDeviceSynchronize(), "hw_blstats_aggregator_create");
    *out = a.release();
    return HW_OK;
}

int hw_blstats_aggregator_destroy(hw_blstats_aggregator* a)
{
    if (!a) return HW_OK;
    cudaFree(a->acc);
    delete a;
    return HW_OK;
}

int hw_blstats_aggregator_add(hw_blstats_aggregator* a, const hw_baseliner_stats* d_stats, hw_frame_interval fi,
                              void* stream)
{
    if (!a || !d_stats) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    const bool aEmpty = a->fi.lower == a->fi.upper, bEmpty = fi.lower == fi.upper;
    if (!aEmpty && !bEmpty && a->fi.upper != fi.lower)
        return Fail(HW_ERR_FRAME_ORDER, "baseliner metrics are not adjacent to the aggregated frame interval");
    HW_CUDA(LaunchAggMerge(a->acc, d_stats, (int)a->lanes, S(stream)), "hw_blstats_aggregator_add");
    if (aEmpty) a->fi = fi;
    else if (!bEmpty) a->fi = hw_frame_interval{std::min(a->fi.lower, fi.lower), std::max(a->fi.upper, fi.upper)};
    return HW_OK;
}

int hw_blstats_aggregator_get(const hw_blstats_aggregator* a, hw_baseliner_stats* d_out, hw_frame_interval* fi,
                              void* stream)
{
    if (!a || !d_out) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(cudaMemcpyAsync(d_out, a->acc, sizeof(hw_baseliner_stats) * a->lanes, cudaMemcpyDeviceToDevice, S(stream)),
            "hw_blstats_aggregator_get");
    if (fi) *fi = a->fi;
    return HW_OK;
}

int hw_blstats_aggregator_reset(hw_blstats_aggregator* a, void* stream)
{
    if (!a) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(LaunchAggReset(a->acc, (int)a->lanes, S(stream)), "hw_blstats_aggregator_reset");
    a->fi = hw_frame_interval{0, 0};
    return HW_OK;
}

// ---- Histogram ---------------------------------------------------------------

int hw_histogram_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, hw_histogram** out)
{
    if (!out) return Fail(HW_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto h = std::make_unique<hw_histogram>();
    int rc = PrepareConfig(cfg, &h->d, &h->k);
    if (rc) return rc;
    if (lanes == 0) return Fail(HW_ERR_INVALID_ARG, "lanes must be positive");
    h->cfg = *cfg;
    h->poolId = pool_id;
    h->lanes = lanes;
    const size_t nZmw = (size_t)lanes * kLane;
    if ((rc = DevAlloc(&h->hist, lanes, "hw_histogram_create"))) return rc;
    if ((rc = DevAlloc(&h->edgePrev, nZmw, "hw_histogram_create"))) return rc;
    if ((rc = DevAlloc(&h->edgeBits, nZmw, "hw_histogram_create"))) return rc;
    if ((rc = DevAlloc(&h->err, 1, "hw_histogram_create"))) return rc;
    HW_CUDA(cudaMemset(h->hist, 0, sizeof(hw_lane_histogram) * lanes), "hw_histogram_create");
    HW_CUDA(cudaMemset(h->edgePrev, 0, nZmw * sizeof(int16_t)), "hw_histogram_create");
    HW_CUDA(cudaMemset(h->edgeBits, 0, nZmw), "hw_histogram_create");
    HW_CUDA(cudaMemset(h->err, 0, sizeof(int)), "hw_histogram_create");
    *out = h.release();
    return HW_OK;
}

int hw_histogram_destroy(hw_histogram* h)
{
    if (!h) return HW_OK;
    cudaFree(h->hist);
    cudaFree(h->edgePrev);
    cudaFree(h->edgeBits);
    cudaFree(h->err);
    delete h;
    return HW_OK;
}

int hw_histogram_add_batch(hw_histogram* h, const int16_t* d_traces, uint32_t frames, hw_frame_interval fi,
                           const hw_lane_model* d_models, void* stream)
{
    if (!h || !d_traces || !d_models) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (!h->initialized)
        return Fail(HW_ERR_NOT_INITIALIZED, "Cannot aggregate trace data into histograms before calling Reset with the desired histogram bounds");
    const bool aEmpty = h->fi.lower == h->fi.upper, bEmpty = fi.lower == fi.upper;
    if (!aEmpty && !bEmpty && h->fi.upper != fi.lower)
        return Fail(HW_ERR_FRAME_ORDER, "trace batch is not adjacent to the histogram's frame interval");
    HW_CUDA(LaunchHistAdd(h->hist, h->edgePrev, h->edgeBits, d_traces, (int)frames, d_models, (int)h->lanes, S(stream)),
            "hw_histogram_add_batch");
    if (aEmpty) h->fi = fi;
    else if (!bEmpty) h->fi = hw_frame_interval{std::min(h->fi.lower, fi.lower), std::max(h->fi.upper, fi.upper)};
    return HW_OK;
}

int hw_histogram_reset_from_stats(hw_histogram* h, const hw_baseliner_stats* d_stats, void* stream)
{
    if (!h || !d_stats) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(LaunchHistResetStats(h->hist, d_stats, (int)h->lanes, h->k, h->err, S(stream)), "hw_histogram_reset_from_stats");
    h->initialized = true;
    h->fi = hw_frame_interval{0, 0};
    int e = TakeDeviceError(h->err, S(stream), "hw_histogram_reset_from_stats");
    if (e) return Fail(e, "UHistogramSimd: lowerBound must be less than upperBound and bins must not underflow");
    return HW_OK;
}

int hw_histogram_reset_from_bounds(hw_histogram* h, const hw_lane_hist_bounds* d_bounds, void* stream)
{
    if (!h || !d_bounds) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(LaunchHistResetBounds(h->hist, d_bounds, (int)h->lanes, h->err, S(stream)), "hw_histogram_reset_from_bounds");
    h->initialized = true;
    h->fi = hw_frame_interval{0, 0};
    int e = TakeDeviceError(h->err, S(stream), "hw_histogram_reset_from_bounds");
    if (e) return Fail(e, "UHistogramSimd: lowerBound must be less than upperBound and bins must not underflow");
    return HW_OK;
}

int hw_histogram_get(const hw_histogram* h, hw_lane_histogram* d_out, hw_frame_interval* fi, void* stream)
{
    if (!h || !d_out) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(cudaMemcpyAsync(d_out, h->hist, sizeof(hw_lane_histogram) * h->lanes, cudaMemcpyDeviceToDevice, S(stream)),
            "hw_histogram_get");
    if (fi) *fi = h->fi;
    return HW_OK;
}

// ---- DME -----------------------------------------------------------------------

int hw_dme_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, hw_dme** out)
{
    if (!out) return Fail(HW_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto d = std::make_unique<hw_dme>();
    int rc = PrepareConfig(cfg, &d->d, &d->k);
    if (rc) return rc;
    if (lanes == 0) return Fail(HW_ERR_INVALID_ARG, "lanes must be positive");
    d->cfg = *cfg;
    d->poolId = pool_id;
    d->lanes = lanes;
    if ((rc = DevAlloc(&d->scratch, (size_t)lanes * 3 * (kBins + 1) * kLane, "hw_dme_create"))) return rc;
    if ((rc = DevAlloc(&d->err, 1, "hw_dme_create"))) return rc;
    HW_CUDA(cudaMemset(d->err, 0, sizeof(int)), "hw_dme_create");
    *out = d.release();
    return HW_OK;
}

int hw_dme_destroy(hw_dme* d)
{
    if (!d) return HW_OK;
    cudaFree(d->scratch);
    cudaFree(d->err);
    cudaFree(d->phases);
    delete d;
    return HW_OK;
}

int hw_dme_profile_phases(hw_dme* d, int enable)
{
    if (!d) return Fail(HW_ERR_INVALID_ARG, "NULL handle");
    if (enable && !d->phases)
    {
        int rc = DevAlloc(&d->phases, (size_t)d->lanes * 8, "hw_dme_profile_phases");
        if (rc) return rc;
        HW_CUDA(cudaMemset(d->phases, 0, (size_t)d->lanes * 8 * sizeof(long long)), "hw_dme_profile_phases");
    }
    else if (!enable && d->phases)
    {
        cudaFree(d->phases);
        d->phases = nullptr;
    }
    return HW_OK;
}

int hw_dme_phase_cycles(const hw_dme* d, int64_t* host_out, void* stream)
{
    if (!d || !host_out) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (!d->phases) return Fail(HW_ERR_INVALID_ARG, "hw_dme_phase_cycles: phase profiling is off");
    HW_CUDA(cudaMemcpyAsync(host_out, d->phases, (size_t)d->lanes * 8 * sizeof(long long), cudaMemcpyDeviceToHost,
                            S(stream)), "hw_dme_phase_cycles");
    HW_CUDA(cudaStreamSynchronize(S(stream)), "hw_dme_phase_cycles");
    return HW_OK;
}

int hw_dme_init_models(hw_dme* d, const hw_baseliner_stats* d_stats, hw_lane_model* d_models, void* stream)
{
    if (!d || !d_stats || !d_models) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(LaunchInitModels(d_models, d_stats, (int)d->lanes, d->k, S(stream)), "hw_dme_init_models");
    return HW_OK;
}

int hw_dme_estimate(hw_dme* d, const hw_lane_histogram* d_hist, const hw_baseliner_stats* d_stats,
                    hw_frame_interval hist_fi, hw_frame_interval model_fi, hw_lane_model* d_models,
                    hw_dme_diag* d_diag, void* stream)
{
    if (!d || !d_hist || !d_stats || !d_models) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (hist_fi.lower == hist_fi.upper || model_fi.lower == model_fi.upper)
        return Fail(HW_ERR_INVALID_ARG, "frame intervals must not be empty");
    DmeArgs a{d_hist, d_stats, d_models, d_diag, d->scratch, d->err, (int)d->lanes,
              model_fi.lower + (model_fi.upper - model_fi.lower) / 2,
              hist_fi.lower + (hist_fi.upper - hist_fi.lower) / 2};
    a.phases = d->phases;
    HW_CUDA(LaunchDmeEstimate(a, d->k, S(stream)), "hw_dme_estimate");
    int e = TakeDeviceError(d->err, S(stream), "hw_dme_estimate");
    if (e) return Fail(e, "DME: a reference sanity assertion failed (non-finite estimate or bad SNR-drop threshold)");
    return HW_OK;
}

int hw_dme_estimate_proposal(hw_dme* d, const hw_lane_histogram* d_hist, const hw_baseliner_stats* d_stats,
                             hw_frame_interval hist_fi, hw_frame_interval model_fi, hw_lane_model* d_models,
                             hw_dme_diag* d_diag, const float* d_proposal, void* stream)
{
    if (!d || !d_hist || !d_stats || !d_models || !d_proposal) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (hist_fi.lower == hist_fi.upper || model_fi.lower == model_fi.upper)
        return Fail(HW_ERR_INVALID_ARG, "frame intervals must not be empty");
    DmeArgs a{d_hist, d_stats, d_models, d_diag, d->scratch, d->err, (int)d->lanes,
              model_fi.lower + (model_fi.upper - model_fi.lower) / 2,
              hist_fi.lower + (hist_fi.upper - hist_fi.lower) / 2, d_proposal};
    a.phases = d->phases;
    HW_CUDA(LaunchDmeEstimate(a, d->k, S(stream)), "hw_dme_estimate_proposal");
    int e = TakeDeviceError(d->err, S(stream), "hw_dme_estimate_proposal");
    if (e) return Fail(e, "DME: a reference sanity assertion failed (non-finite estimate or bad SNR-drop threshold)");
    return HW_OK;
}

// ---- Frame labeler ---------------------------------------------------------------

int hw_labeler_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, uint32_t frames_per_chunk,
                      hw_labeler** out)
{
    if (!out) return Fail(HW_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto l = std::make_unique<hw_labeler>();
    int rc = PrepareConfig(cfg, &l->d, &l->k);
    if (rc) return rc;
    if (lanes == 0) return Fail(HW_ERR_INVALID_ARG, "lanes must be positive");
    if (frames_per_chunk < (uint32_t)(kLatent + kLookback) || frames_per_chunk > 1024)
        return Fail(HW_ERR_INVALID_ARG, "frames_per_chunk must be in [40, 1024]");
    l->cfg = *cfg;
    l->poolId = pool_id;
    l->lanes = lanes;
    l->F = frames_per_chunk;
    const size_t nZmw = (size_t)lanes * kLane;
    if ((rc = DevAlloc(&l->latModel, lanes, "hw_labeler_create"))) return rc;
    if ((rc = DevAlloc(&l->latLabel, nZmw, "hw_labeler_create"))) return rc;
    if ((rc = DevAlloc(&l->latRoi, nZmw, "hw_labeler_create"))) return rc;
    if ((rc = DevAlloc(&l->latTrc, nZmw, "hw_labeler_create"))) return rc;
    if ((rc = DevAlloc(&l->prevLat, (size_t)kLatent * nZmw, "hw_labeler_create"))) return rc;
    if ((rc = DevAlloc(&l->tb, (size_t)(frames_per_chunk + kLookback) * nZmw, "hw_labeler_create"))) return rc;
    HW_CUDA(cudaMemset(l->latLabel, 0, nZmw * 2), "hw_labeler_create");
    HW_CUDA(cudaMemset(l->latRoi, 0, nZmw * 2), "hw_labeler_create");
    HW_CUDA(cudaMemset(l->latTrc, 0, nZmw * 2), "hw_labeler_create");
    HW_CUDA(cudaMemset(l->prevLat, 0, (size_t)kLatent * nZmw * 2), "hw_labeler_create");
    // LatentViterbi ctor (FrameLabelerHost.cpp:58-70): baseline N(0, 50), analogs N(1000, 10).
    std::vector<hw_lane_model> m(lanes);
    std::memset(m.data(), 0, sizeof(hw_lane_model) * lanes);
    for (auto& lm : m)
        for (int z = 0; z < kLane; ++z)
        {
            lm.baseline.means[z] = f32_to_f16_bits(0.0f);
            lm.baseline.vars[z] = f32_to_f16_bits(50.0f);
            for (int a = 0; a < kAnalogs; ++a)
            {
                lm.analogs[a].means[z] = f32_to_f16_bits(1000.0f);
                lm.analogs[a].vars[z] = f32_to_f16_bits(10.0f);
            }
        }
    HW_CUDA(cudaMemcpy(l->latModel, m.data(), sizeof(hw_lane_model) * lanes, cudaMemcpyHostToDevice), "hw_labeler_create");
    *out = l.release();
    return HW_OK;
}

int hw_labeler_destroy(hw_labeler* l)
{
    if (!l) return HW_OK;
    cudaFree(l->latModel);
    cudaFree(l->latLabel);
    cudaFree(l->latRoi);
    cudaFree(l->latTrc);
    cudaFree(l->prevLat);
    cudaFree(l->tb);
    cudaFree(l->gap);
    delete l;
    return HW_OK;
}

int hw_labeler_process(hw_labeler* l, const int16_t* d_traces, const hw_lane_model* d_models, int16_t* d_labels,
                       int16_t* d_latent_out, float* d_viterbi_score, float* d_margin_or_null, void* stream)
{
    if (!l || !d_traces || !d_models || !d_labels) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (d_margin_or_null && !l->gap)
    {
        int rc = DevAlloc(&l->gap, (size_t)l->lanes * (l->F + hwp::kViterbiStitchLookback) * kStates * kLane,
                          "hw_labeler_process (margin scratch)");
        if (rc) return rc;
    }
    LabelerArgs a{d_traces, d_models, d_labels, d_latent_out, d_viterbi_score, l->latModel, l->latLabel, l->latRoi,
                  l->latTrc, l->prevLat, l->tb, (int)l->lanes, (int)l->F};
    a.margin = d_margin_or_null;
    a.gap = l->gap;
    HW_CUDA(LaunchLabeler(a, l->k, S(stream)), "hw_labeler_process");
    return HW_OK;
}

// ---- Pulse accumulator -----------------------------------------------------------

int hw_pulse_accumulator_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, uint32_t frames_per_chunk,
                                hw_pulse_accumulator** out)
{
    if (!out) return Fail(HW_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto p = std::make_unique<hw_pulse_accumulator>();
    int rc = PrepareConfig(cfg, &p->d, &p->k);
    if (rc) return rc;
    if (lanes == 0 || frames_per_chunk < (uint32_t)kLatent) return Fail(HW_ERR_INVALID_ARG, "bad lanes or frames_per_chunk");
    p->cfg = *cfg;
    p->poolId = pool_id;
    p->lanes = lanes;
    p->F = frames_per_chunk;
    const size_t nZmw = (size_t)lanes * kLane;
    if ((rc = DevAlloc(&p->segStart, nZmw, "hw_pulse_accumulator_create"))) return rc;
    if ((rc = DevAlloc(&p->segFirst, nZmw, "hw_pulse_accumulator_create"))) return rc;
    if ((rc = DevAlloc(&p->segLast, nZmw, "hw_pulse_accumulator_create"))) return rc;
    if ((rc = DevAlloc(&p->segMax, nZmw, "hw_pulse_accumulator_create"))) return rc;
    if ((rc = DevAlloc(&p->segTotal, nZmw, "hw_pulse_accumulator_create"))) return rc;
    if ((rc = DevAlloc(&p->segM2, nZmw, "hw_pulse_accumulator_create"))) return rc;
    if ((rc = DevAlloc(&p->segLabel, nZmw, "hw_pulse_accumulator_create"))) return rc;
    HW_CUDA(cudaMemset(p->segStart, 0, nZmw * 4), "hw_pulse_accumulator_create");
    HW_CUDA(cudaMemset(p->segFirst, 0, nZmw * 2), "hw_pulse_accumulator_create");
    HW_CUDA(cudaMemset(p->segLast, 0, nZmw * 2), "hw_pulse_accumulator_create");
    HW_CUDA(cudaMemset(p->segMax, 0, nZmw * 2), "hw_pulse_accumulator_create");
    HW_CUDA(cudaMemset(p->segTotal, 0, nZmw * 4), "hw_pulse_accumulator_create");
    HW_CUDA(cudaMemset(p->segM2, 0, nZmw * 4), "hw_pulse_accumulator_create");
    HW_CUDA(cudaMemset(p->segLabel, 0, nZmw * 2), "hw_pulse_accumulator_create");
    *out = p.release();
    return HW_OK;
}

int hw_pulse_accumulator_destroy(hw_pulse_accumulator* p)
{
    if (!p) return HW_OK;
    cudaFree(p->segStart); cudaFree(p->segFirst); cudaFree(p->segLast); cudaFree(p->segMax);
    cudaFree(p->segTotal); cudaFree(p->segM2); cudaFree(p->segLabel);
    delete p;
    return HW_OK;
}

int hw_pulse_accumulator_process(hw_pulse_accumulator* p, const int16_t* d_labels, const int16_t* d_latent_trace,
                                 const int16_t* d_trace, int32_t first_frame, const hw_lane_model* d_models,
                                 hw_pulse* d_pulses, uint32_t* d_lens, uint32_t* d_overflows,
                                 hw_stat_accum_state* d_blstats, void* stream)
{
    if (!p || !d_labels || !d_latent_trace || !d_trace || !d_models || !d_pulses || !d_lens || !d_overflows || !d_blstats)
        return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    PulseArgs a{d_labels, d_latent_trace, d_trace, d_models, d_pulses, d_lens, d_overflows, d_blstats,
                p->segStart, p->segFirst, p->segLast, p->segMax, p->segTotal, p->segM2, p->segLabel,
                (int)p->lanes, (int)p->F, (uint32_t)first_frame};
    HW_CUDA(LaunchPulses(a, p->k, S(stream)), "hw_pulse_accumulator_process");
    return HW_OK;
}

}   // extern "C"

// ---- Batch analyzer ------------------------------------------------------------
// BatchAnalyzer (analyzer/BatchAnalyzer.cpp:149-375) with the
// DetectionModelEstimator state machine (DetectionModelEstimator.cpp:93-160).
// All stages of a chunk are enqueued on one stream; the aggregated statistics
// and the histogram are read in place by the model kernels.

struct hw_analyzer
{
    enum Status { HIST_INIT = 0, DME_INIT = 1, SEQUENCING = 2 };
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    uint32_t poolId = 0, lanes = 0, F = 0;
    hw_baseliner* bl = nullptr;
    hw_blstats_aggregator* agg = nullptr;
    hw_histogram* hist = nullptr;
    hw_dme* dme = nullptr;
    hw_labeler* lab = nullptr;
    hw_pulse_accumulator* pa = nullptr;
    int16_t* bls = nullptr;
    hw_baseliner_stats* stats = nullptr;
    hw_lane_model* models = nullptr;
    int16_t* labels = nullptr;
    int16_t* latent = nullptr;
    float* score = nullptr;
    hw_stat_accum_state* paStats = nullptr;
    hw_dme_diag* diag = nullptr;
    bool diagValid = false;
    // learned EM start (hw_analyzer_set_learned_init), not owned
    hw_learned_init* net = nullptr;
    float* lProp = nullptr;     // [lanes][15][64]
    hw_frame_interval modelFi{0, 0};
    int status = HIST_INIT;
    int32_t framesRemaining = 0;
    bool initialized = false;
    bool fullEstimation = false;
    uint32_t blLatency = 0;
    int32_t poolDelay = 0;
    int32_t nextFrame = 0;
    // Stage timers (AnalysisProfiler counterpart, TA/AnalysisProfiler.h):
    // event pairs recorded around each stage while profiling is enabled.
    bool profiling = false;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    std::vector<std::pair<int, size_t>> evMarks;   // (stage, index of start event)

    cudaEvent_t NextEvent()
    {
        if (evUsed == evPool.size())
        {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
            evPool.push_back(e);
        }
        return evPool[evUsed++];
    }
    size_t Begin(int stage, cudaStream_t s)
    {
        if (!profiling) return 0;
        const size_t i = evUsed;
        cudaEvent_t e0 = NextEvent(), e1 = NextEvent();
        if (!e0 || !e1) return 0;
        cudaEventRecord(e0, s);
        evMarks.emplace_back(stage, i);
        return i + 1;
    }
    void End(size_t tok, cudaStream_t s)
    {
        if (tok) cudaEventRecord(evPool[tok], s);
    }

    ~hw_analyzer()
    {
        for (auto e : evPool) cudaEventDestroy(e);
        hw_baseliner_destroy(bl);
        hw_blstats_aggregator_destroy(agg);
        hw_histogram_destroy(hist);
        hw_dme_destroy(dme);
        hw_labeler_destroy(lab);
        hw_pulse_accumulator_destroy(pa);
        cudaFree(bls); cudaFree(stats); cudaFree(models); cudaFree(labels); cudaFree(latent);
        cudaFree(score); cudaFree(paStats); cudaFree(diag);
        cudaFree(lProp);
    }

    // DetectionModelEstimator::AddBatch
    int DmeAdd(hw_frame_interval fi, cudaStream_t s, bool* ran)
    {
        int rc;
        *ran = false;
        size_t t = Begin(HW_STAGE_AGGREGATE, s);
        if ((rc = hw_blstats_aggregator_add(agg, stats, fi, s))) return rc;
        End(t, s);
        if (status != HIST_INIT)
        {
            t = Begin(HW_STAGE_HISTOGRAM, s);
            if ((rc = hw_histogram_add_batch(hist, bls, F, fi, models, s))) return rc;
            End(t, s);
        }
        if (status != SEQUENCING)
        {
            t = Begin(HW_STAGE_MODEL_INIT, s);
            if ((rc = hw_dme_init_models(dme, agg->acc, models, s))) return rc;
            End(t, s);
            modelFi = agg->fi;
        }
        framesRemaining -= (int32_t)F;
        if (framesRemaining <= 0)
        {
            if (status == DME_INIT) status = SEQUENCING;
            if (status == SEQUENCING)
            {
                *ran = true;
                t = Begin(HW_STAGE_DME, s);
                if (net)
                {
                    if ((rc = hw_learned_init_propose(net, lanes, hist->hist, agg->acc, lProp, s))) return rc;
                    if ((rc = hw_dme_estimate_proposal(dme, hist->hist, agg->acc, hist->fi, modelFi, models, diag,
                                                       lProp, s))) return rc;
                }
                else if ((rc = hw_dme_estimate(dme, hist->hist, agg->acc, hist->fi, modelFi, models, diag, s))) return rc;
                End(t, s);
                diagValid = true;
                modelFi = hist->fi;
            }
            t = Begin(HW_STAGE_HIST_RESET, s);
            if ((rc = hw_histogram_reset_from_stats(hist, agg->acc, s))) return rc;
            if ((rc = hw_blstats_aggregator_reset(agg, s))) return rc;
            End(t, s);
            if (status == HIST_INIT) status = DME_INIT;
            framesRemaining = (int32_t)cfg.min_frames_for_estimate;
        }
        return HW_OK;
    }

    int LabelAndPulse(int32_t ff, hw_pulse* pulses, uint32_t* lens, uint32_t* ovf, cudaStream_t s)
    {
        int rc;
        size_t t = Begin(HW_STAGE_LABELER, s);
        if ((rc = hw_labeler_process(lab, bls, models, labels, latent, score, nullptr, s))) return rc;
        End(t, s);
        t = Begin(HW_STAGE_PULSES, s);
        // The labels batch starts hw_labeler_latent_frames() before the trace
        // chunk (LabelsBatchFactory::NewBatch, LabelsBatch.h:112-121).
        rc = hw_pulse_accumulator_process(pa, labels, latent, bls, ff - (int32_t)hwp::kLatentFrames, models, pulses,
                                          lens, ovf, paStats, s);
        End(t, s);
        return rc;
    }
};

extern "C" {

int hw_analyzer_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, uint32_t frames_per_chunk,
                       hw_analyzer** out)
{
    if (!out) return Fail(HW_ERR_INVALID_ARG, "out is NULL");
    *out = nullptr;
    auto a = std::make_unique<hw_analyzer>();
    int rc = PrepareConfig(cfg, &a->d, &a->k);
    if (rc) return rc;
    a->cfg = *cfg;
    a->poolId = pool_id;
    a->lanes = lanes;
    a->F = frames_per_chunk;
    if ((rc = hw_baseliner_create(cfg, pool_id, lanes, frames_per_chunk, &a->bl))) return rc;
    if ((rc = hw_blstats_aggregator_create(pool_id, lanes, &a->agg))) return rc;
    if ((rc = hw_histogram_create(cfg, pool_id, lanes, &a->hist))) return rc;
    if ((rc = hw_dme_create(cfg, pool_id, lanes, &a->dme))) return rc;
    if ((rc = hw_labeler_create(cfg, pool_id, lanes, frames_per_chunk, &a->lab))) return rc;
    if ((rc = hw_pulse_accumulator_create(cfg, pool_id, lanes, frames_per_chunk, &a->pa))) return rc;
    const size_t nZmw = (size_t)lanes * kLane;
    if ((rc = DevAlloc(&a->bls, nZmw * frames_per_chunk, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->stats, lanes, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->models, lanes, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->labels, nZmw * frames_per_chunk, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->latent, nZmw * kLatent, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->score, nZmw, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->paStats, lanes, "hw_analyzer_create"))) return rc;
    if ((rc = DevAlloc(&a->diag, lanes, "hw_analyzer_create"))) return rc;
    HW_CUDA(cudaMemset(a->models, 0, sizeof(hw_lane_model) * lanes), "hw_analyzer_create");
    if (cfg->model_estimation_mode == HW_FIXED_ESTIMATIONS)
    {
        // FixedModelBatchAnalyzer: the static model in every lane, from the start
        hw_lane_model m;
        hwp::StaticModel(*cfg, &m);
        std::vector<hw_lane_model> host(lanes, m);
        HW_CUDA(cudaMemcpy(a->models, host.data(), sizeof(hw_lane_model) * lanes, cudaMemcpyHostToDevice),
                "hw_analyzer_create");
    }
    a->framesRemaining = (int32_t)cfg->num_frames_pre_accum_stats;
    a->blLatency = a->d.baselinerStartupLatency;
    const uint32_t chunksPerEstimate = (std::max(cfg->min_frames_for_estimate, 1u) + frames_per_chunk - 1) / frames_per_chunk;
    a->poolDelay = (int32_t)((pool_id % chunksPerEstimate) * frames_per_chunk);
    *out = a.release();
    return HW_OK;
}

int hw_analyzer_set_learned_init(hw_analyzer* a, hw_learned_init* net)
{
    if (!a) return Fail(HW_ERR_INVALID_ARG, "NULL analyzer");
    if (net && !a->lProp)
    {
        const int rc = DevAlloc(&a->lProp, (size_t)a->lanes * 15 * kLane, "hw_analyzer_set_learned_init");
        if (rc) return rc;
    }
    a->net = net;
    return HW_OK;
}

// ---- Checkpoints -----------------------------------------------------------------
// The blob is a header (sizes, the schedule state kept on the host) followed
// by every device buffer that carries state from one chunk to the next, in
// a fixed order.  Per-chunk outputs and scratch are not saved.

namespace {

struct StateHeader
{
    char magic[8];
    uint32_t version, lanes, F, poolId;
    int32_t filterType, estimationMode;
    uint64_t payload;
    int32_t status, framesRemaining, initialized, fullEstimation, nextFrame, diagValid;
    hw_frame_interval modelFi, aggFi, histFi;
    int32_t histInitialized, pad_;
};

const char kStateMagic[8] = {'H', 'W', 'B', '2', '0', '0', 'S', 'T'};

std::vector<std::pair<void*, size_t>> StateSegments(const hw_analyzer* a)
{
    const size_t n = (size_t)a->lanes * kLane;
    return {
        {a->bl->st16, (size_t)a->bl->slots16 * n * sizeof(int16_t)},
        {a->bl->st32, 3 * n * sizeof(float)},
        {a->agg->acc, a->lanes * sizeof(hw_baseliner_stats)},
        {a->hist->hist, a->lanes * sizeof(hw_lane_histogram)},
        {a->hist->edgePrev, n * sizeof(int16_t)},
        {a->hist->edgeBits, n * sizeof(uint8_t)},
        {a->lab->latModel, a->lanes * sizeof(hw_lane_model)},
        {a->lab->latLabel, n * sizeof(int16_t)},
        {a->lab->latRoi, n * sizeof(int16_t)},
        {a->lab->latTrc, n * sizeof(int16_t)},
        {a->lab->prevLat, (size_t)kLatent * n * sizeof(int16_t)},
        {a->pa->segStart, n * sizeof(uint32_t)},
        {a->pa->segFirst, n * sizeof(int16_t)},
        {a->pa->segLast, n * sizeof(int16_t)},
        {a->pa->segMax, n * sizeof(int16_t)},
        {a->pa->segTotal, n * sizeof(float)},
        {a->pa->segM2, n * sizeof(float)},
        {a->pa->segLabel, n * sizeof(int16_t)},
        {a->models, a->lanes * sizeof(hw_lane_model)},
        {a->diag, a->lanes * sizeof(hw_dme_diag)},
    };
}

uint64_t StatePayload(const hw_analyzer* a)
{
    uint64_t t = 0;
    for (const auto& seg : StateSegments(a)) t += seg.second;
    return t;
}

}   // namespace

int hw_analyzer_state_size(const hw_analyzer* a, uint64_t* bytes)
{
    if (!a || !bytes) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    *bytes = sizeof(StateHeader) + StatePayload(a);
    return HW_OK;
}

int hw_analyzer_state_export(const hw_analyzer* a, void* host_blob, uint64_t bytes, void* stream)
{
    if (!a || !host_blob) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    const uint64_t payload = StatePayload(a);
    if (bytes < sizeof(StateHeader) + payload) return Fail(HW_ERR_INVALID_ARG, "state blob too small");
    StateHeader h{};
    memcpy(h.magic, kStateMagic, 8);
    h.version = 1;
    h.lanes = a->lanes;
    h.F = a->F;
    h.poolId = a->poolId;
    h.filterType = a->cfg.filter_type;
    h.estimationMode = a->cfg.model_estimation_mode;
    h.payload = payload;
    h.status = a->status;
    h.framesRemaining = a->framesRemaining;
    h.initialized = a->initialized;
    h.fullEstimation = a->fullEstimation;
    h.nextFrame = a->nextFrame;
    h.diagValid = a->diagValid;
    h.modelFi = a->modelFi;
    h.aggFi = a->agg->fi;
    h.histFi = a->hist->fi;
    h.histInitialized = a->hist->initialized;
    char* out = static_cast<char*>(host_blob);
    memcpy(out, &h, sizeof(h));
    size_t off = sizeof(h);
    cudaStream_t s = S(stream);
    for (const auto& seg : StateSegments(a))
    {
        HW_CUDA(cudaMemcpyAsync(out + off, seg.first, seg.second, cudaMemcpyDeviceToHost, s), "hw_analyzer_state_export");
        off += seg.second;
    }
    HW_CUDA(cudaStreamSynchronize(s), "hw_analyzer_state_export");
    return HW_OK;
}

int hw_analyzer_state_import(hw_analyzer* a, const void* host_blob, uint64_t bytes, void* stream)
{
    if (!a || !host_blob) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (bytes < sizeof(StateHeader)) return Fail(HW_ERR_INVALID_ARG, "state blob too small");
    StateHeader h;
    memcpy(&h, host_blob, sizeof(h));
    if (memcmp(h.magic, kStateMagic, 8) != 0 || h.version != 1)
        return Fail(HW_ERR_INVALID_ARG, "not an hw_analyzer state blob of version 1");
    if (h.lanes != a->lanes || h.F != a->F || h.poolId != a->poolId || h.filterType != a->cfg.filter_type ||
        h.estimationMode != a->cfg.model_estimation_mode)
        return Fail(HW_ERR_INVALID_ARG, "state blob is for a different pool, size, filter or estimation mode");
    const uint64_t payload = StatePayload(a);
    if (h.payload != payload || bytes < sizeof(h) + payload)
        return Fail(HW_ERR_INVALID_ARG, "state blob size does not match this analyzer");
    const char* in = static_cast<const char*>(host_blob);
    size_t off = sizeof(h);
    cudaStream_t s = S(stream);
    for (const auto& seg : StateSegments(a))
    {
        HW_CUDA(cudaMemcpyAsync(seg.first, in + off, seg.second, cudaMemcpyHostToDevice, s), "hw_analyzer_state_import");
        off += seg.second;
    }
    HW_CUDA(cudaStreamSynchronize(s), "hw_analyzer_state_import");
    a->status = h.status;
    a->framesRemaining = h.framesRemaining;
    a->initialized = h.initialized != 0;
    a->fullEstimation = h.fullEstimation != 0;
    a->nextFrame = h.nextFrame;
    a->diagValid = h.diagValid != 0;
    a->modelFi = h.modelFi;
    a->agg->fi = h.aggFi;
    a->hist->fi = h.histFi;
    a->hist->initialized = h.histInitialized != 0;
    return HW_OK;
}

int hw_analyzer_destroy(hw_analyzer* a)
{
    delete a;
    return HW_OK;
}

static int AnalyzerProcess(hw_analyzer* a, const int16_t* d_trace, const uint8_t* d_trace8, int32_t first_frame,
                           hw_pulse* d_pulses, uint32_t* d_lens, uint32_t* d_overflows, int32_t* emitted,
                           int32_t* estimated, void* stream)
{
    if (!a || !(d_trace || d_trace8) || !d_pulses || !d_lens || !d_overflows)
        return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (first_frame != a->nextFrame) return Fail(HW_ERR_FRAME_ORDER, "Bad frame ID.");
    cudaStream_t s = S(stream);
    int rc;
    bool ran = false, emit = false;
    const size_t nZmw = (size_t)a->lanes * kLane;
    {
        const size_t t = a->Begin(HW_STAGE_BASELINE, s);
        if ((rc = d_trace8 ? hw_baseliner_process_u8(a->bl, d_trace8, first_frame, a->bls, a->stats, s)
                           : hw_baseliner_process(a->bl, d_trace, first_frame, a->bls, a->stats, s))) return rc;
        a->End(t, s);
    }
    const hw_frame_interval fi{first_frame, first_frame + (int32_t)a->F};
    if (a->cfg.model_estimation_mode == HW_FIXED_ESTIMATIONS)
    {
        // FixedModelBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:172-207)
        if ((rc = a->LabelAndPulse(first_frame, d_pulses, d_lens, d_overflows, s))) return rc;
        emit = true;
    }
    else if (a->cfg.model_estimation_mode == HW_INITIAL_ESTIMATIONS)
    {
        // SingleEstimateBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:177-256)
        if (!a->initialized && first_frame > (int32_t)a->blLatency)
        {
            if ((rc = a->DmeAdd(fi, s, &ran))) return rc;
            a->initialized = ran;
        }
        if (a->initialized)
        {
            if ((rc = a->LabelAndPulse(first_frame, d_pulses, d_lens, d_overflows, s))) return rc;
            emit = true;
        }
    }
    else
    {
        // DynamicEstimateBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:289-375)
        if (first_frame >= (int32_t)a->blLatency + a->poolDelay)
        {
            if ((rc = a->DmeAdd(fi, s, &ran))) return rc;
            if (ran) a->fullEstimation = true;
            if ((rc = a->LabelAndPulse(first_frame, d_pulses, d_lens, d_overflows, s))) return rc;
            emit = a->fullEstimation;
        }
    }
    if (!emit)
    {
        HW_CUDA(cudaMemsetAsync(d_lens, 0, nZmw * sizeof(uint32_t), s), "hw_analyzer_process");
        HW_CUDA(cudaMemsetAsync(d_overflows, 0, nZmw * sizeof(uint32_t), s), "hw_analyzer_process");
    }
    a->nextFrame = first_frame + (int32_t)a->F;
    if (emitted) *emitted = emit ? 1 : 0;
    if (estimated) *estimated = ran ? 1 : 0;
    return HW_OK;
}

int hw_analyzer_process(hw_analyzer* a, const int16_t* d_trace, int32_t first_frame, hw_pulse* d_pulses,
                        uint32_t* d_lens, uint32_t* d_overflows, int32_t* emitted, int32_t* estimated, void* stream)
{
    const hwk::NvtxRange range("hw_analyzer_process");
    return AnalyzerProcess(a, d_trace, nullptr, first_frame, d_pulses, d_lens, d_overflows, emitted, estimated, stream);
}

int hw_analyzer_process_u8(hw_analyzer* a, const uint8_t* d_trace, int32_t first_frame, hw_pulse* d_pulses,
                           uint32_t* d_lens, uint32_t* d_overflows, int32_t* emitted, int32_t* estimated,
                           void* stream)
{
    return AnalyzerProcess(a, nullptr, d_trace, first_frame, d_pulses, d_lens, d_overflows, emitted, estimated, stream);
}

int hw_analyzer_models(const hw_analyzer* a, hw_lane_model* d_out, hw_frame_interval* fi, void* stream)
{
    if (!a || !d_out) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    HW_CUDA(cudaMemcpyAsync(d_out, a->models, sizeof(hw_lane_model) * a->lanes, cudaMemcpyDeviceToDevice, S(stream)),
            "hw_analyzer_models");
    if (fi) *fi = a->modelFi;
    return HW_OK;
}

int hw_analyzer_chunk_metrics(const hw_analyzer* a, hw_baseliner_stats* d_baseliner_stats, float* d_viterbi_score,
                              hw_stat_accum_state* d_pd_baseline_stats, void* stream)
{
    if (!a) return Fail(HW_ERR_INVALID_ARG, "NULL analyzer");
    cudaStream_t s = S(stream);
    if (d_baseliner_stats)
        HW_CUDA(cudaMemcpyAsync(d_baseliner_stats, a->stats, sizeof(hw_baseliner_stats) * a->lanes,
                                cudaMemcpyDeviceToDevice, s), "hw_analyzer_chunk_metrics");
    if (d_viterbi_score)
        HW_CUDA(cudaMemcpyAsync(d_viterbi_score, a->score, sizeof(float) * a->lanes * kLane, cudaMemcpyDeviceToDevice, s),
                "hw_analyzer_chunk_metrics");
    if (d_pd_baseline_stats)
        HW_CUDA(cudaMemcpyAsync(d_pd_baseline_stats, a->paStats, sizeof(hw_stat_accum_state) * a->lanes,
                                cudaMemcpyDeviceToDevice, s), "hw_analyzer_chunk_metrics");
    return HW_OK;
}

int hw_analyzer_last_diag(const hw_analyzer* a, hw_dme_diag* d_out, int32_t* valid, void* stream)
{
    if (!a || !d_out) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (valid) *valid = a->diagValid ? 1 : 0;
    if (!a->diagValid) return HW_OK;
    HW_CUDA(cudaMemcpyAsync(d_out, a->diag, sizeof(hw_dme_diag) * a->lanes, cudaMemcpyDeviceToDevice, S(stream)),
            "hw_analyzer_last_diag");
    return HW_OK;
}

int hw_analyzer_profile(hw_analyzer* a, int32_t enable)
{
    if (!a) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    a->profiling = enable != 0;
    return HW_OK;
}

int hw_analyzer_stage_times(hw_analyzer* a, double ms[HW_NUM_STAGES], uint32_t launches[HW_NUM_STAGES])
{
    if (!a || !ms || !launches) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    for (int i = 0; i < HW_NUM_STAGES; ++i) { ms[i] = 0.0; launches[i] = 0; }
    for (const auto& m : a->evMarks)
    {
        HW_CUDA(cudaEventSynchronize(a->evPool[m.second + 1]), "hw_analyzer_stage_times");
        float t = 0.0f;
        HW_CUDA(cudaEventElapsedTime(&t, a->evPool[m.second], a->evPool[m.second + 1]), "hw_analyzer_stage_times");
        ms[m.first] += t;
        launches[m.first] += 1;
    }
    a->evMarks.clear();
    a->evUsed = 0;
    return HW_OK;
}

}   // extern "C"

// ---- Pool sets: uneven pools in shared launches ---------------------------------
// Lanes are independent through the whole chain, and a pool's estimation
// schedule depends only on its chunk length F and its stagger class
// pool_id % chunksPerEstimate (BatchAnalyzer.cpp:96-117).  Pools that share
// both are therefore run as one batched analyzer over all their lanes: each
// stage is one launch for the whole class, with results identical to
// separate per-pool analyzers.  The packed input holds the classes one after
// the other, so every class's chunk is one contiguous slice.

struct hw_pool_set
{
    struct Group
    {
        hw_analyzer* an = nullptr;
        uint32_t lanes = 0, F = 0;
        uint64_t inOffset = 0;                // int16 elements into the packed chunk
        hw_pulse* pulses = nullptr;
        uint32_t* lens = nullptr;
        uint32_t* ovf = nullptr;
        std::vector<uint32_t> pools;
    };
    uint32_t cap = 0;
    std::vector<Group> groups;
    std::vector<uint32_t> poolGroup, poolLaneOffset;
    std::vector<uint64_t> poolInOffset;
    uint64_t total = 0;

    ~hw_pool_set()
    {
        for (auto& g : groups)
        {
            hw_analyzer_destroy(g.an);
            cudaFree(g.pulses); cudaFree(g.lens); cudaFree(g.ovf);
        }
    }
};

extern "C" {

int hw_pool_set_create(const hw_config* cfg, uint32_t n_pools, const uint32_t* lanes, const uint32_t* frames_per_chunk,
                       hw_pool_set** out)
{
    if (!cfg || !lanes || !frames_per_chunk || !out || n_pools == 0) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    *out = nullptr;
    auto ps = std::make_unique<hw_pool_set>();
    ps->cap = cfg->max_calls_per_zmw;
    ps->poolGroup.assign(n_pools, 0);
    ps->poolLaneOffset.assign(n_pools, 0);
    ps->poolInOffset.assign(n_pools, 0);
    // class key: (F, stagger class); classes in order of first appearance
    std::vector<std::pair<uint32_t, uint32_t>> keys;
    for (uint32_t p = 0; p < n_pools; ++p)
    {
        if (lanes[p] == 0) return Fail(HW_ERR_INVALID_ARG, "every pool needs at least one lane");
        const uint32_t F = frames_per_chunk[p];
        if (F == 0) return Fail(HW_ERR_INVALID_ARG, "frames_per_chunk must be positive");
        const uint32_t cpe = (std::max(cfg->min_frames_for_estimate, 1u) + F - 1) / F;
        const std::pair<uint32_t, uint32_t> key{F, p % cpe};
        size_t gi = 0;
        while (gi < keys.size() && keys[gi] != key) ++gi;
        if (gi == keys.size())
        {
            keys.push_back(key);
            ps->groups.emplace_back();
            ps->groups.back().F = F;
        }
        auto& g = ps->groups[gi];
        ps->poolGroup[p] = (uint32_t)gi;
        ps->poolLaneOffset[p] = g.lanes;
        g.lanes += lanes[p];
        g.pools.push_back(p);
    }
    uint64_t off = 0;
    for (auto& g : ps->groups)
    {
        g.inOffset = off;
        for (uint32_t p : g.pools) ps->poolInOffset[p] = off + (uint64_t)ps->poolLaneOffset[p] * g.F * kLane;
        off += (uint64_t)g.lanes * g.F * kLane;
        int rc = hw_analyzer_create(cfg, g.pools.front(), g.lanes, g.F, &g.an);
        if (rc) return rc;
        const size_t n = (size_t)g.lanes * kLane;
        if ((rc = DevAlloc(&g.pulses, n * ps->cap, "hw_pool_set_create"))) return rc;
        if ((rc = DevAlloc(&g.lens, n, "hw_pool_set_create"))) return rc;
        if ((rc = DevAlloc(&g.ovf, n, "hw_pool_set_create"))) return rc;
    }
    ps->total = off;
    *out = ps.release();
    return HW_OK;
}

int hw_pool_set_destroy(hw_pool_set* s)
{
    delete s;
    return HW_OK;
}

int hw_pool_set_layout(const hw_pool_set* s, uint64_t* in_offsets, uint64_t* total_elements, uint32_t* n_launch_groups)
{
    if (!s) return Fail(HW_ERR_INVALID_ARG, "NULL pool set");
    if (in_offsets)
        for (size_t p = 0; p < s->poolInOffset.size(); ++p) in_offsets[p] = s->poolInOffset[p];
    if (total_elements) *total_elements = s->total;
    if (n_launch_groups) *n_launch_groups = (uint32_t)s->groups.size();
    return HW_OK;
}

int hw_pool_set_process(hw_pool_set* s, const int16_t* d_packed, int32_t step, int32_t* emitted, int32_t* estimated,
                        void* stream)
{
    if (!s || !d_packed || step < 0) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    for (auto& g : s->groups)
    {
        int32_t em = 0, est = 0;
        int rc = hw_analyzer_process(g.an, d_packed + g.inOffset, step * (int32_t)g.F, g.pulses, g.lens, g.ovf, &em,
                                     &est, stream);
        if (rc) return rc;
        for (uint32_t p : g.pools)
        {
            if (emitted) emitted[p] = em;
            if (estimated) estimated[p] = est;
        }
    }
    return HW_OK;
}

int hw_pool_set_outputs(const hw_pool_set* s, uint32_t pool, hw_pulse** d_pulses, uint32_t** d_lens,
                        uint32_t** d_overflows)
{
    if (!s || pool >= s->poolGroup.size()) return Fail(HW_ERR_INVALID_ARG, "bad pool");
    const auto& g = s->groups[s->poolGroup[pool]];
    const size_t z0 = (size_t)s->poolLaneOffset[pool] * kLane;
    if (d_pulses) *d_pulses = g.pulses + z0 * s->cap;
    if (d_lens) *d_lens = g.lens + z0;
    if (d_overflows) *d_overflows = g.ovf + z0;
    return HW_OK;
}

}   // extern "C"
