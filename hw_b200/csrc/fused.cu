// Fused chunk engine: every pool of a basecaller in one handle, each stage of
// a chunk step one launch over a list of lanes (hw_chunk_fused).
//
// The reference runs one BatchAnalyzer per pool and chunk
// (AN/BatchAnalyzer.cpp:119-375, AN = src/basecaller/basecaller/analyzer),
// each of its filters launching over that pool's lanes.  Here the state of
// all pools is packed lane after lane; per step the host walks every pool's
// schedule (the DetectionModelEstimator state machine,
// TA/DetectionModelEstimator.cpp:93-160, and the Fixed / SingleEstimate /
// DynamicEstimate analyzers, AN/BatchAnalyzer.cpp:172-375) and appends the
// pool's lanes to the list of every stage it takes.  The lists go to the
// device with one copy each and every stage runs once over its list, so a
// step is about a dozen launches however many pools there are and however
// uneven they are.  Nothing in a step waits for the device: device-detected
// failures travel back through a pinned word read two steps later.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "hw_device.cuh"

using namespace hwk;

namespace {

int Fail(int code, const std::string& msg) { return hwk::SetLastError(code, msg.c_str()); }

#define HWF_CUDA(expr, where)                                                                     \
    do {                                                                                          \
        cudaError_t e_ = (expr);                                                                  \
        if (e_ != cudaSuccess) return Fail(HW_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
int Alloc(T** p, size_t count, const char* where)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
    if (e != cudaSuccess) return Fail(HW_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
    return HW_OK;
}

template <typename T>
int AllocZero(T** p, size_t count, const char* where)
{
    int rc = Alloc(p, count, where);
    if (rc) return rc;
    HWF_CUDA(cudaMemset(*p, 0, std::max<size_t>(count, 1) * sizeof(T)), where);
    return HW_OK;
}

// The stage lists of one step, in launch order.
enum List
{
    L_BASE16,     // baseline filter, int16 chunks
    L_BASE8,      // baseline filter, uint8 chunks
    L_AGG,        // BaselineStatsAggregator::AddMetrics
    L_HIST,       // TraceHistogramAccumulator::AddBatch
    L_INIT,       // CoreDMEstimator::InitDetectionModels
    L_DME,        // CoreDMEstimator::Estimate
    L_RESET,      // histogram reset from the aggregated statistics + aggregator reset
    L_LABEL1,     // frame labeler + pulse accumulator, separate kernels, 1/2/4 lanes a labeler block
    L_LABEL2,
    L_LABEL4,
    L_LP1,        // frame labeler + pulse accumulator in one kernel, 1/2/4 lanes a block
    L_LP2,
    L_LP4,
    L_LABEL1L,    // the same six for pools that run the DME this step (after it)
    L_LABEL2L,
    L_LABEL4L,
    L_LP1L,
    L_LP2L,
    L_LP4L,
    L_HF,         // HF metrics filter
    L_ZERO,       // pools that emit nothing this step
    kNumLists
};

int LanesPerCta(int list) { return 1 << ((list - L_LABEL1) % 3); }
bool FusedPulses(int list) { return (list - L_LABEL1) % 6 >= 3; }

// Per pool: hw_analyzer's schedule state.
struct PoolRt
{
    enum Status { HIST_INIT = 0, DME_INIT = 1, SEQUENCING = 2 };
    uint32_t id = 0, lanes = 0, F = 0, lane0 = 0;
    int status = HIST_INIT;
    int32_t framesRemaining = 0;
    bool initialized = false, fullEstimation = false, histInitialized = false, diagValid = false;
    int32_t blLatency = 0, poolDelay = 0, nextFrame = 0;
    hw_frame_interval modelFi{0, 0}, aggFi{0, 0}, histFi{0, 0};
    uint32_t hfSeen = 0;      // HFMetricsFilter::framesSeen_
};

hw_frame_interval Merge(hw_frame_interval a, hw_frame_interval b)
{
    const bool aEmpty = a.lower == a.upper, bEmpty = b.lower == b.upper;
    if (aEmpty) return b;
    if (bEmpty) return a;
    return hw_frame_interval{std::min(a.lower, b.lower), std::max(a.upper, b.upper)};
}

int32_t Center(hw_frame_interval fi) { return fi.lower + (fi.upper - fi.lower) / 2; }

// Step tables reach the device through a kernel that reads the pinned host
// copy directly (not a copy-engine transfer, which would queue behind the
// caller's large chunk uploads and hold up the analysis stream).
constexpr int kMaxSegs = 1 + kNumLists;
struct TableCopy
{
    const uint32_t* src[kMaxSegs];
    uint32_t* dst[kMaxSegs];
    uint32_t words[kMaxSegs];
    int n;
};

__global__ void TableCopyKernel(TableCopy t)
{
    const uint32_t stride = gridDim.x * blockDim.x;
    for (int i = 0; i < t.n; ++i)
        for (uint32_t w = blockIdx.x * blockDim.x + threadIdx.x; w < t.words[i]; w += stride) t.dst[i][w] = t.src[i][w];
}

// The device failure word goes back the same way, into pinned host memory.
__global__ void ErrorOutKernel(const int* err, int* hostErr)
{
    if (threadIdx.x == 0) *hostErr = *err;
}

}   // namespace

struct hw_fused
{
    hw_config cfg;
    hwp::Derived d;
    KParams k;
    std::vector<PoolRt> pools;
    uint32_t lanes = 0;
    int maxF = 0;
    // tuning per chunk length: {fuse label+pulses, labeler lanes per block}
    std::map<uint32_t, std::pair<uint32_t, uint32_t>> tuning;

    // device state, packed over the engine's lanes
    int16_t* st16 = nullptr;
    float* st32 = nullptr;
    hw_baseliner_stats* stats = nullptr;
    hw_baseliner_stats* acc = nullptr;
    hw_lane_histogram* hist = nullptr;
    int16_t* edgePrev = nullptr;
    uint8_t* edgeBits = nullptr;
    hw_lane_model* models = nullptr;
    hw_dme_diag* diag = nullptr;
    float* dmeScratch = nullptr;      // [launch lane][3][kBins + 1][64]
    uint32_t dmeCap = 0;              // launch lanes the scratch holds
    hw_lane_model* latModel = nullptr;
    int16_t* latLabel = nullptr;
    int16_t* latRoi = nullptr;
    int16_t* latTrc = nullptr;
    int16_t* prevLat = nullptr;
    uint32_t* tb = nullptr;
    int16_t* bls = nullptr;
    int16_t* labels = nullptr;
    int16_t* latent = nullptr;
    float* score = nullptr;
    hw_stat_accum_state* paStats = nullptr;
    uint32_t* segStart = nullptr;
    int16_t* segFirst = nullptr;
    int16_t* segLast = nullptr;
    int16_t* segMax = nullptr;
    float* segTotal = nullptr;
    float* segM2 = nullptr;
    int16_t* segLabel = nullptr;
    int* err = nullptr;

    // HF metrics filter (hw_fused_enable_hf_metrics)
    bool hf = false;
    uint32_t hfBlock = 4096;
    float hfFrameRate = 100.0f;
    int hfRealtime = 1;
    void* hfState = nullptr;
    int16_t* hfLeft = nullptr;
    int16_t* hfRight = nullptr;
    int8_t* hfFeature = nullptr;
    float* hfThr = nullptr;
    int8_t* hfValue = nullptr;
    int hfNodes = 0;
    float hfHsw[2] = {0, 0}, hfMaxHsw = 0;

    // lane tables and the per-step tables (pinned host copies, two in flight)
    int32_t* dPoolOf = nullptr;
    uint64_t* dFrameOff = nullptr;
    PoolStep* dSteps = nullptr;
    int32_t* dLists = nullptr;        // [kNumLists][lanes]
    PoolStep* hSteps[2] = {nullptr, nullptr};
    int32_t* hLists[2] = {nullptr, nullptr};
    int* hErr[2] = {nullptr, nullptr};
    // device addresses of the three pinned host buffers
    PoolStep* mSteps[2] = {nullptr, nullptr};
    int32_t* mLists[2] = {nullptr, nullptr};
    int* mErr[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    bool inFlight[2] = {false, false};
    uint64_t step = 0;
    int sticky = HW_OK;

    // CUDA graphs per step plan, captured on a stream of the engine's own
    // (the caller's stream may be the legacy default stream, which cannot be
    // captured) and replayed on the caller's stream
    bool graphs = false;
    cudaStream_t capStream = nullptr;
    // a second stream for the statistics merge, histogram, DME and reset,
    // beside the main stream's initialisation and labeling (see Launch)
    cudaStream_t side = nullptr;
    cudaEvent_t evFork = nullptr, evHist = nullptr, evInit = nullptr, evJoin = nullptr;
    int overlapMode = 1;              // hw_fused_set_overlap
    // learned EM start (hw_fused_set_learned_init), not owned: the proposal
    // of each estimating pool is written to lProp [lane][15][64] before the DME
    hw_learned_init* net = nullptr;
    float* lProp = nullptr;
    std::vector<int> dmePools;        // pools that run the DME this step
    std::map<std::vector<int64_t>, cudaGraphExec_t> graphCache;
    std::map<std::vector<int64_t>, int> planSeen;
    uint32_t lastLaunches = 0, lastGraphLaunches = 0;

    // Stage timers (as hw_analyzer_profile): event pairs around each stage's
    // launches while profiling; steps are not replayed from graphs meanwhile.
    bool profiling = false;
    std::vector<cudaEvent_t> evPool;
    size_t evUsed = 0;
    std::vector<std::pair<int, size_t>> evMarks;   // (stage, index of start event)
    size_t Begin(int stage, cudaStream_t s)
    {
        if (!profiling) return 0;
        while (evPool.size() < evUsed + 2)
        {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return 0;
            evPool.push_back(e);
        }
        const size_t i = evUsed;
        evUsed += 2;
        cudaEventRecord(evPool[i], s);
        evMarks.emplace_back(stage, i);
        return i + 1;
    }
    void End(size_t tok, cudaStream_t s)
    {
        if (tok) cudaEventRecord(evPool[tok], s);
    }

    ~hw_fused()
    {
        for (auto& g : graphCache) cudaGraphExecDestroy(g.second);
        for (auto e : evPool) cudaEventDestroy(e);
        if (capStream) cudaStreamDestroy(capStream);
        if (side) cudaStreamDestroy(side);
        if (evFork) cudaEventDestroy(evFork);
        if (evHist) cudaEventDestroy(evHist);
        if (evInit) cudaEventDestroy(evInit);
        if (evJoin) cudaEventDestroy(evJoin);
        for (int b = 0; b < 2; ++b)
        {
            if (ev[b]) cudaEventDestroy(ev[b]);
            cudaFreeHost(hSteps[b]);
            cudaFreeHost(hLists[b]);
            cudaFreeHost(hErr[b]);
        }
        void* bufs[] = {st16, st32, stats, acc, hist, edgePrev, edgeBits, models, diag, dmeScratch, latModel,
                        latLabel, latRoi, latTrc, prevLat, tb, bls, labels, latent, score, paStats, segStart,
                        segFirst, segLast, segMax, segTotal, segM2, segLabel, err, dPoolOf, dFrameOff, dSteps,
                        dLists, hfState, hfLeft, hfRight, hfFeature, hfThr, hfValue, lProp};
        for (void* p : bufs) cudaFree(p);
    }

    int Launch(cudaStream_t s, const int32_t counts[kNumLists], const int maxFList[kNumLists], uint32_t* launches);
    int Schedule(hw_pool_chunk* table, int b, int32_t counts[kNumLists], int maxFList[kNumLists]);
};

// Walks every pool's schedule for this step (host state only) and fills the
// stage lists and per-pool step records of buffer b.
int hw_fused::Schedule(hw_pool_chunk* table, int b, int32_t counts[kNumLists], int maxFList[kNumLists])
{
    for (int s = 0; s < kNumLists; ++s) { counts[s] = 0; maxFList[s] = 0; }
    dmePools.clear();
    int32_t* lists = hLists[b];
    const int minFrames = (int)cfg.min_frames_for_estimate;
    for (size_t p = 0; p < pools.size(); ++p)
    {
        PoolRt& P = pools[p];
        hw_pool_chunk& c = table[p];
        const int32_t ff = c.first_frame;
        PoolStep& st = hSteps[b][p];
        st = PoolStep{c.d_trace, c.d_trace8, c.d_pulses, c.d_lens, c.d_overflows, ff, (int32_t)P.F, (int32_t)P.lane0,
                      0, 0, 0, c.d_metrics};
        auto append = [&](int s) {
            int32_t* dst = lists + (size_t)s * lanes + counts[s];
            for (uint32_t i = 0; i < P.lanes; ++i) dst[i] = (int32_t)(P.lane0 + i);
            counts[s] += (int32_t)P.lanes;
            maxFList[s] = std::max(maxFList[s], (int)P.F);
        };
        append(c.d_trace8 ? L_BASE8 : L_BASE16);
        const hw_frame_interval fi{ff, ff + (int32_t)P.F};
        bool ran = false, emit = false;
        // DetectionModelEstimator::AddBatch (DetectionModelEstimator.cpp:93-160)
        auto dmeAdd = [&]() -> int {
            append(L_AGG);
            P.aggFi = Merge(P.aggFi, fi);
            if (P.status != PoolRt::HIST_INIT)
            {
                if (!P.histInitialized)
                    return Fail(HW_ERR_NOT_INITIALIZED, "histogram used before its bounds were set");
                append(L_HIST);
                P.histFi = Merge(P.histFi, fi);
            }
            if (P.status != PoolRt::SEQUENCING)
            {
                append(L_INIT);
                P.modelFi = P.aggFi;
            }
            P.framesRemaining -= (int32_t)P.F;
            if (P.framesRemaining <= 0)
            {
                if (P.status == PoolRt::DME_INIT) P.status = PoolRt::SEQUENCING;
                if (P.status == PoolRt::SEQUENCING)
                {
                    if (P.histFi.lower == P.histFi.upper || P.modelFi.lower == P.modelFi.upper)
                        return Fail(HW_ERR_INVALID_ARG, "frame intervals must not be empty");
                    ran = true;
                    st.tModel = Center(P.modelFi);
                    st.tEst = Center(P.histFi);
                    append(L_DME);
                    dmePools.push_back((int)p);
                    P.diagValid = true;
                    P.modelFi = P.histFi;
                }
                append(L_RESET);
                P.histInitialized = true;
                P.histFi = hw_frame_interval{0, 0};
                P.aggFi = hw_frame_interval{0, 0};
                if (P.status == PoolRt::HIST_INIT) P.status = PoolRt::DME_INIT;
                P.framesRemaining = minFrames;
            }
            return HW_OK;
        };
        auto labelAndPulse = [&]() {
            // kernel choice of this chunk length (default: separate kernels, 2 lanes a block)
            uint32_t fuse = 0, lpc = 2;
            auto t = tuning.find(P.F);
            if (t != tuning.end()) { fuse = t->second.first; lpc = t->second.second; }
            // a pool whose models the DME replaces this step is labeled after
            // it; the others' labeling may overlap the DME
            append((ran ? L_LABEL1L : L_LABEL1) + (fuse ? 3 : 0) + (lpc == 1 ? 0 : lpc == 2 ? 1 : 2));
        };
        int rc = HW_OK;
        if (cfg.model_estimation_mode == HW_FIXED_ESTIMATIONS)
        {
            // FixedModelBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:172-207)
            labelAndPulse();
            emit = true;
        }
        else if (cfg.model_estimation_mode == HW_INITIAL_ESTIMATIONS)
        {
            // SingleEstimateBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:177-256)
            if (!P.initialized && ff > P.blLatency)
            {
                if ((rc = dmeAdd())) return rc;
                P.initialized = ran;
            }
            if (P.initialized)
            {
                labelAndPulse();
                emit = true;
            }
        }
        else
        {
            // DynamicEstimateBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:289-375)
            if (ff >= P.blLatency + P.poolDelay)
            {
                if ((rc = dmeAdd())) return rc;
                if (ran) P.fullEstimation = true;
                labelAndPulse();
                emit = P.fullEstimation;
            }
        }
        if (!emit) append(L_ZERO);
        // HF metrics (BatchAnalyzer.cpp:201, 278, 368): every chunk for the
        // fixed-model and single-estimate analyzers -- before the first
        // estimate on an empty pulse batch with zero scores --, only emitting
        // chunks for the dynamic one.  The pulse batch is the labels batch,
        // 24 latent frames before the trace chunk.
        c.metrics_emitted = 0;
        if (hf)
        {
            const bool labeled = (cfg.model_estimation_mode == HW_FIXED_ESTIMATIONS)
                              || (cfg.model_estimation_mode == HW_INITIAL_ESTIMATIONS ? P.initialized : emit);
            const bool runs = cfg.model_estimation_mode != HW_DYNAMIC_ESTIMATIONS || emit;
            if (runs)
            {
                const int64_t last = (int64_t)ff - kLatent + P.F;
                const bool finalize = (uint32_t)(last % (int64_t)hfBlock) < P.F;
                st.hfFlags = (P.hfSeen == 0 ? kHfReset : 0) | (finalize ? kHfFinalize : 0) | (labeled ? 0 : kHfEmpty);
                P.hfSeen = finalize ? 0 : P.hfSeen + P.F;
                c.metrics_emitted = finalize ? 1 : 0;
                append(L_HF);
            }
        }
        P.nextFrame = ff + (int32_t)P.F;
        c.emitted = emit ? 1 : 0;
        c.estimated = ran ? 1 : 0;
    }
    return HW_OK;
}

// Enqueues the step's kernels over the device lists (also what a graph captures).
int hw_fused::Launch(cudaStream_t s, const int32_t counts[kNumLists], const int maxFList[kNumLists],
                     uint32_t* launches)
{
    uint32_t n = 0;
    auto map = [&](int l) {
        LaneMap m;
        m.list = dLists + (size_t)l * lanes;
        m.n = counts[l];
        m.poolOf = dPoolOf;
        m.frameOff = dFrameOff;
        m.pools = dSteps;
        return m;
    };
    const int L = (int)lanes;
    for (int l : {L_BASE16, L_BASE8})
        if (counts[l])
        {
            BaselinerArgs a{nullptr, bls, stats, st16, st32, L, maxFList[l]};
            a.map = map(l);
            a.u8 = l == L_BASE8;
            const size_t t = Begin(HW_STAGE_BASELINE, s);
            HWF_CUDA(LaunchBaseliner(cfg.filter_type, a, k, s), "hw_chunk_fused: baseline filter");
            End(t, s);
            ++n;
        }
    auto doAgg = [&](cudaStream_t st) -> int {
        if (!counts[L_AGG]) return HW_OK;
        const size_t t = Begin(HW_STAGE_AGGREGATE, st);
        HWF_CUDA(LaunchAggMerge(acc, stats, L, st, map(L_AGG)), "hw_chunk_fused: statistics merge");
        End(t, st);
        ++n;
        return HW_OK;
    };
    auto doHist = [&](cudaStream_t st) -> int {
        if (!counts[L_HIST]) return HW_OK;
        const size_t t = Begin(HW_STAGE_HISTOGRAM, st);
        HWF_CUDA(LaunchHistAdd(hist, edgePrev, edgeBits, bls, maxFList[L_HIST], models, L, st, map(L_HIST)),
                 "hw_chunk_fused: histogram");
        End(t, st);
        ++n;
        return HW_OK;
    };
    auto doInit = [&](cudaStream_t st) -> int {
        if (!counts[L_INIT]) return HW_OK;
        const size_t t = Begin(HW_STAGE_MODEL_INIT, st);
        HWF_CUDA(LaunchInitModels(models, acc, L, k, st, map(L_INIT)), "hw_chunk_fused: model initialisation");
        End(t, st);
        ++n;
        return HW_OK;
    };
    auto doDme = [&](cudaStream_t st) -> int {
        if (!counts[L_DME]) return HW_OK;
        DmeArgs a{hist, acc, models, diag, dmeScratch, err, L, 0, 0};
        a.map = map(L_DME);
        const size_t t = Begin(HW_STAGE_DME, st);
        if (net)
        {
            // the network's proposal for each estimating pool's lanes (the
            // DME reads it by engine lane), then the learned-start estimate
            for (int p : dmePools)
            {
                const PoolRt& P = pools[p];
                const int prc = hw_learned_init_propose(net, P.lanes, hist + P.lane0, acc + P.lane0,
                                                        lProp + (size_t)P.lane0 * 15 * kLane, st);
                if (prc) return prc;
                ++n;
            }
            a.proposal = lProp;
        }
        HWF_CUDA(LaunchDmeEstimate(a, k, st), "hw_chunk_fused: DME");
        End(t, st);
        ++n;
        return HW_OK;
    };
    auto doReset = [&](cudaStream_t st) -> int {
        if (!counts[L_RESET]) return HW_OK;
        const size_t t = Begin(HW_STAGE_HIST_RESET, st);
        HWF_CUDA(LaunchHistResetStats(hist, acc, L, k, err, st, map(L_RESET)), "hw_chunk_fused: histogram reset");
        HWF_CUDA(LaunchAggReset(acc, L, st, map(L_RESET)), "hw_chunk_fused: aggregator reset");
        End(t, st);
        n += 2;
        return HW_OK;
    };
    // Labeling of one list (+ the pulse accumulator, fused or after it).
    auto label = [&](int l, cudaStream_t st) -> int {
        if (!counts[l]) return HW_OK;
        const bool fuse = FusedPulses(l);
        LabelerArgs la{bls, models, labels, latent, score, latModel, latLabel, latRoi, latTrc, prevLat, tb, L,
                       maxFList[l]};
        la.map = map(l);
        PulseArgs pa{labels, latent, bls, models, nullptr, nullptr, nullptr, paStats, segStart, segFirst, segLast,
                     segMax, segTotal, segM2, segLabel, L, maxFList[l], 0};
        pa.map = map(l);
        size_t t = Begin(HW_STAGE_LABELER, st);
        HWF_CUDA(LaunchLabeler(la, k, st, fuse ? &pa : nullptr, LanesPerCta(l)), "hw_chunk_fused: labeler");
        End(t, st);
        n += 2;
        if (!fuse)
        {
            t = Begin(HW_STAGE_PULSES, st);
            HWF_CUDA(LaunchPulses(pa, k, st), "hw_chunk_fused: pulse accumulator");
            End(t, st);
            ++n;
        }
        return HW_OK;
    };
    int rc;
    const int ov = overlapMode;
    if (profiling || ov == 0)
    {
        // one stream in the reference's order (the stage timers time one stream)
        if ((rc = doAgg(s)) || (rc = doHist(s)) || (rc = doInit(s)) || (rc = doDme(s)) || (rc = doReset(s))) return rc;
        for (int l = L_LABEL1; l <= L_LP4L; ++l)
            if ((rc = label(l, s))) return rc;
    }
    else if (ov == 1)
    {
        // Merge, histogram and initialisation in order; with a DME this step,
        // the DME and reset run on the side stream beside the labeling of the
        // pools without an estimate, and the estimating pools are labeled
        // after them.
        if ((rc = doAgg(s)) || (rc = doHist(s)) || (rc = doInit(s))) return rc;
        int early = 0;
        for (int l = L_LABEL1; l <= L_LP4; ++l) early += counts[l] ? 1 : 0;
        if (counts[L_DME] && early)
        {
            HWF_CUDA(cudaEventRecord(evFork, s), "hw_chunk_fused: fork");
            HWF_CUDA(cudaStreamWaitEvent(side, evFork, 0), "hw_chunk_fused: fork");
            if ((rc = doDme(side)) || (rc = doReset(side))) return rc;
            HWF_CUDA(cudaEventRecord(evJoin, side), "hw_chunk_fused: join");
            for (int l = L_LABEL1; l <= L_LP4; ++l)
                if ((rc = label(l, s))) return rc;
            HWF_CUDA(cudaStreamWaitEvent(s, evJoin, 0), "hw_chunk_fused: join");
        }
        else
        {
            if ((rc = doDme(s)) || (rc = doReset(s))) return rc;
            for (int l = L_LABEL1; l <= L_LP4; ++l)
                if ((rc = label(l, s))) return rc;
        }
        for (int l = L_LABEL1L; l <= L_LP4L; ++l)
            if ((rc = label(l, s))) return rc;
    }
    else
    {
        // The histogram beside the labeling too.  Side:
        // statistics merge, histogram, DME, histogram reset.  Main: model
        // initialisation, then the labeling of the pools without an
        // estimate, beside the side stream's work; the estimating pools are
        // labeled after it.  Orderings kept from the single-stream sequence:
        // the histogram reads the models before the initialisation writes
        // them and the initialisation reads the merged statistics (main waits
        // for the histogram when it initialises); the DME of a pool
        // initialised this step reads its new models and the reset clears
        // statistics the initialisation read (side waits for the
        // initialisation); labeling reads the DME's models (main waits for
        // the side stream before the estimating pools' labeling).
        HWF_CUDA(cudaEventRecord(evFork, s), "hw_chunk_fused: fork");
        HWF_CUDA(cudaStreamWaitEvent(side, evFork, 0), "hw_chunk_fused: fork");
        if ((rc = doAgg(side)) || (rc = doHist(side))) return rc;
        HWF_CUDA(cudaEventRecord(evHist, side), "hw_chunk_fused: fork");
        if (counts[L_INIT])
        {
            HWF_CUDA(cudaStreamWaitEvent(s, evHist, 0), "hw_chunk_fused: fork");
            if ((rc = doInit(s))) return rc;
        }
        HWF_CUDA(cudaEventRecord(evInit, s), "hw_chunk_fused: fork");
        HWF_CUDA(cudaStreamWaitEvent(side, evInit, 0), "hw_chunk_fused: fork");
        if ((rc = doDme(side)) || (rc = doReset(side))) return rc;
        HWF_CUDA(cudaEventRecord(evJoin, side), "hw_chunk_fused: join");
        for (int l = L_LABEL1; l <= L_LP4; ++l)
            if ((rc = label(l, s))) return rc;
        HWF_CUDA(cudaStreamWaitEvent(s, evJoin, 0), "hw_chunk_fused: join");
        for (int l = L_LABEL1L; l <= L_LP4L; ++l)
            if ((rc = label(l, s))) return rc;
    }
    if (counts[L_HF])
    {
        HfEngineArgs a{};
        a.map = map(L_HF);
        a.state = hfState;
        a.cap = (int)cfg.max_calls_per_zmw;
        a.bs = stats;
        a.models = models;
        a.viterbi = score;
        a.pd = paStats;
        a.realtime = hfRealtime;
        a.frameRate = hfFrameRate;
        a.left = hfLeft; a.right = hfRight; a.feature = hfFeature; a.thr = hfThr; a.value = hfValue;
        a.nodes = hfNodes;
        a.hsw0 = hfHsw[0]; a.hsw1 = hfHsw[1]; a.maxHsw = hfMaxHsw;
        const size_t t = Begin(HW_STAGE_METRICS, s);
        HWF_CUDA(LaunchHfMapped(a, s), "hw_chunk_fused: HF metrics");
        End(t, s);
        ++n;
    }
    if (counts[L_ZERO])
    {
        HWF_CUDA(LaunchZeroOutputs(map(L_ZERO), s), "hw_chunk_fused: empty outputs");
        ++n;
    }
    *launches = n;
    return HW_OK;
}

namespace {

const char* kDeferredMsg =
    "a device-side check failed in an earlier step (histogram bounds, UHistogramSimd.cpp:66-96, or a DME sanity "
    "assertion); the analysis cannot continue";

// Collects the failure word of buffer b's step once that step has finished.
int Collect(hw_fused* f, int b)
{
    if (!f->inFlight[b]) return HW_OK;
    HWF_CUDA(cudaEventSynchronize(f->ev[b]), "hw_chunk_fused");
    f->inFlight[b] = false;
    if (*f->hErr[b] != 0 && f->sticky == HW_OK) f->sticky = *f->hErr[b];
    return HW_OK;
}

}   // namespace

extern "C" {

int hw_fused_create(const hw_config* cfg, uint32_t n_pools, const uint32_t* pool_ids, const uint32_t* lanes,
                    const uint32_t* frames_per_chunk, hw_fused** out)
{
    if (!cfg || !lanes || !frames_per_chunk || !out || n_pools == 0) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    *out = nullptr;
    auto f = std::make_unique<hw_fused>();
    int rc = hwk::PrepareConfigNoAlloc(cfg, &f->d, &f->k);
    if (rc) return rc;
    f->cfg = *cfg;
    const uint32_t stride = (uint32_t)f->d.aggStride;
    const uint32_t minFrames = std::max(cfg->min_frames_for_estimate, 1u);
    uint64_t total = 0, frameElems = 0;
    std::vector<int32_t> poolOf;
    std::vector<uint64_t> frameOff;
    f->pools.resize(n_pools);
    for (uint32_t p = 0; p < n_pools; ++p)
    {
        const uint32_t F = frames_per_chunk[p];
        if (lanes[p] == 0) return Fail(HW_ERR_INVALID_ARG, "every pool needs at least one lane");
        if (F % stride != 0 || F < (uint32_t)(kLatent + kLookback) || F > 1024)
            return Fail(HW_ERR_INVALID_ARG,
                        "frames_per_chunk must be a multiple of the filter's aggregate stride in [40, 1024]");
        if (total + lanes[p] > (uint64_t)INT32_MAX / kLane) return Fail(HW_ERR_INVALID_ARG, "too many lanes");
        PoolRt& P = f->pools[p];
        P.id = pool_ids ? pool_ids[p] : p;
        P.lanes = lanes[p];
        P.F = F;
        P.lane0 = (uint32_t)total;
        P.framesRemaining = (int32_t)cfg->num_frames_pre_accum_stats;
        P.blLatency = (int32_t)f->d.baselinerStartupLatency;
        const uint32_t chunksPerEstimate = (minFrames + F - 1) / F;
        P.poolDelay = (int32_t)((P.id % chunksPerEstimate) * F);
        for (uint32_t i = 0; i < lanes[p]; ++i)
        {
            poolOf.push_back((int32_t)p);
            frameOff.push_back(frameElems);
            frameElems += (uint64_t)F * kLane;
        }
        total += lanes[p];
        f->maxF = std::max(f->maxF, (int)F);
    }
    const uint32_t L = (uint32_t)total;
    f->lanes = L;
    const size_t nZmw = (size_t)L * kLane;
    const char* where = "hw_fused_create";
    const int slots16 = BaselinerNumSlots16(cfg->filter_type);
    if ((rc = Alloc(&f->st16, (size_t)slots16 * nZmw, where))) return rc;
    if ((rc = Alloc(&f->st32, 3 * nZmw, where))) return rc;
    HWF_CUDA(LaunchBaselinerInit(cfg->filter_type, f->st16, f->st32, (int)L, 0), where);
    if ((rc = AllocZero(&f->stats, L, where))) return rc;
    if ((rc = Alloc(&f->acc, L, where))) return rc;
    HWF_CUDA(LaunchAggReset(f->acc, (int)L, 0), where);
    if ((rc = AllocZero(&f->hist, L, where))) return rc;
    if ((rc = AllocZero(&f->edgePrev, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->edgeBits, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->models, L, where))) return rc;
    if (cfg->model_estimation_mode == HW_FIXED_ESTIMATIONS)
    {
        // FixedModelBatchAnalyzer: the static model in every lane, from the start
        hw_lane_model m;
        hwp::StaticModel(*cfg, &m);
        std::vector<hw_lane_model> host(L, m);
        HWF_CUDA(cudaMemcpy(f->models, host.data(), sizeof(hw_lane_model) * L, cudaMemcpyHostToDevice), where);
    }
    if ((rc = AllocZero(&f->diag, L, where))) return rc;
    if ((rc = Alloc(&f->latModel, L, where))) return rc;
    {
        // LatentViterbi ctor (FrameLabelerHost.cpp:58-70): baseline N(0, 50), analogs N(1000, 10).
        hw_lane_model lm;
        std::memset(&lm, 0, sizeof(lm));
        for (int z = 0; z < kLane; ++z)
        {
            lm.baseline.means[z] = hwm::f32_to_f16_bits(0.0f);
            lm.baseline.vars[z] = hwm::f32_to_f16_bits(50.0f);
            for (int a = 0; a < kAnalogs; ++a)
            {
                lm.analogs[a].means[z] = hwm::f32_to_f16_bits(1000.0f);
                lm.analogs[a].vars[z] = hwm::f32_to_f16_bits(10.0f);
            }
        }
        std::vector<hw_lane_model> host(L, lm);
        HWF_CUDA(cudaMemcpy(f->latModel, host.data(), sizeof(hw_lane_model) * L, cudaMemcpyHostToDevice), where);
    }
    if ((rc = AllocZero(&f->latLabel, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->latRoi, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->latTrc, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->prevLat, (size_t)kLatent * nZmw, where))) return rc;
    if ((rc = Alloc(&f->tb, frameElems + (size_t)kLookback * nZmw, where))) return rc;
    if ((rc = Alloc(&f->bls, frameElems, where))) return rc;
    if ((rc = Alloc(&f->labels, frameElems, where))) return rc;
    if ((rc = AllocZero(&f->latent, (size_t)kLatent * nZmw, where))) return rc;
    if ((rc = AllocZero(&f->score, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->paStats, L, where))) return rc;
    if ((rc = AllocZero(&f->segStart, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->segFirst, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->segLast, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->segMax, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->segTotal, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->segM2, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->segLabel, nZmw, where))) return rc;
    if ((rc = AllocZero(&f->err, 1, where))) return rc;
    if ((rc = Alloc(&f->dPoolOf, L, where))) return rc;
    if ((rc = Alloc(&f->dFrameOff, L, where))) return rc;
    HWF_CUDA(cudaMemcpy(f->dPoolOf, poolOf.data(), L * sizeof(int32_t), cudaMemcpyHostToDevice), where);
    HWF_CUDA(cudaMemcpy(f->dFrameOff, frameOff.data(), L * sizeof(uint64_t), cudaMemcpyHostToDevice), where);
    if ((rc = AllocZero(&f->dSteps, n_pools, where))) return rc;
    if ((rc = AllocZero(&f->dLists, (size_t)kNumLists * L, where))) return rc;
    for (int b = 0; b < 2; ++b)
    {
        // mapped: the step kernels read the tables and write the failure word in place
        HWF_CUDA(cudaHostAlloc((void**)&f->hSteps[b], sizeof(PoolStep) * n_pools, cudaHostAllocMapped), where);
        HWF_CUDA(cudaHostAlloc((void**)&f->hLists[b], sizeof(int32_t) * kNumLists * (size_t)L, cudaHostAllocMapped),
                 where);
        HWF_CUDA(cudaHostAlloc((void**)&f->hErr[b], sizeof(int), cudaHostAllocMapped), where);
        *f->hErr[b] = 0;
        HWF_CUDA(cudaHostGetDevicePointer((void**)&f->mSteps[b], f->hSteps[b], 0), where);
        HWF_CUDA(cudaHostGetDevicePointer((void**)&f->mLists[b], f->hLists[b], 0), where);
        HWF_CUDA(cudaHostGetDevicePointer((void**)&f->mErr[b], f->hErr[b], 0), where);
        HWF_CUDA(cudaEventCreateWithFlags(&f->ev[b], cudaEventDisableTiming), where);
    }
    HWF_CUDA(cudaStreamCreateWithFlags(&f->side, cudaStreamNonBlocking), where);
    HWF_CUDA(cudaEventCreateWithFlags(&f->evFork, cudaEventDisableTiming), where);
    HWF_CUDA(cudaEventCreateWithFlags(&f->evHist, cudaEventDisableTiming), where);
    HWF_CUDA(cudaEventCreateWithFlags(&f->evInit, cudaEventDisableTiming), where);
    HWF_CUDA(cudaEventCreateWithFlags(&f->evJoin, cudaEventDisableTiming), where);
    HWF_CUDA(cudaDeviceSynchronize(), where);
    *out = f.release();
    return HW_OK;
}

int hw_fused_destroy(hw_fused* f)
{
    if (f) cudaDeviceSynchronize();
    delete f;
    return HW_OK;
}

int hw_fused_enable_hf_metrics(hw_fused* f, uint32_t frames_per_block, double frame_rate,
                               int32_t realtime_activity_labels, const int16_t* children_left,
                               const int16_t* children_right, const int8_t* feature, const float* threshold,
                               const int8_t* value, uint32_t n_nodes, const float* hsw_curve,
                               float max_acceptable_halfsandwich_rate)
{
    if (!f || frames_per_block == 0 || !(frame_rate > 0)) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    if (f->step != 0) return Fail(HW_ERR_INVALID_ARG, "HF metrics must be enabled before the first step");
    const bool cart = children_left && children_right && feature && threshold && value && hsw_curve && n_nodes > 0;
    if (cart)
    {
        if (n_nodes > 32767) return Fail(HW_ERR_INVALID_ARG, "too many CART nodes");
        for (uint32_t i = 0; i < n_nodes; ++i)
        {
            if (feature[i] >= 11) return Fail(HW_ERR_INVALID_ARG, "CART feature index out of range");
            if (feature[i] >= 0 && (children_left[i] < 0 || children_left[i] >= (int)n_nodes || children_right[i] < 0 ||
                                    children_right[i] >= (int)n_nodes))
                return Fail(HW_ERR_INVALID_ARG, "CART child index out of range");
        }
    }
    const char* where = "hw_fused_enable_hf_metrics";
    int rc;
    if (!f->hfState)
    {
        const size_t bytes = HfLaneBytes() * f->lanes;
        HWF_CUDA(cudaMalloc(&f->hfState, bytes), where);
        HWF_CUDA(cudaMemset(f->hfState, 0, bytes), where);
        HWF_CUDA(LaunchHfInit(f->hfState, (int)f->lanes, 0), where);
    }
    if (cart)
    {
        cudaFree(f->hfLeft); cudaFree(f->hfRight); cudaFree(f->hfFeature); cudaFree(f->hfThr); cudaFree(f->hfValue);
        f->hfLeft = f->hfRight = nullptr; f->hfFeature = f->hfValue = nullptr; f->hfThr = nullptr;
        if ((rc = Alloc(&f->hfLeft, n_nodes, where))) return rc;
        if ((rc = Alloc(&f->hfRight, n_nodes, where))) return rc;
        if ((rc = Alloc(&f->hfFeature, n_nodes, where))) return rc;
        if ((rc = Alloc(&f->hfThr, n_nodes, where))) return rc;
        if ((rc = Alloc(&f->hfValue, n_nodes, where))) return rc;
        HWF_CUDA(cudaMemcpy(f->hfLeft, children_left, 2 * n_nodes, cudaMemcpyHostToDevice), where);
        HWF_CUDA(cudaMemcpy(f->hfRight, children_right, 2 * n_nodes, cudaMemcpyHostToDevice), where);
        HWF_CUDA(cudaMemcpy(f->hfFeature, feature, n_nodes, cudaMemcpyHostToDevice), where);
        HWF_CUDA(cudaMemcpy(f->hfThr, threshold, 4 * n_nodes, cudaMemcpyHostToDevice), where);
        HWF_CUDA(cudaMemcpy(f->hfValue, value, n_nodes, cudaMemcpyHostToDevice), where);
        f->hfNodes = (int)n_nodes;
        f->hfHsw[0] = hsw_curve[0];
        f->hfHsw[1] = hsw_curve[1];
        f->hfMaxHsw = max_acceptable_halfsandwich_rate;
    }
    HWF_CUDA(cudaDeviceSynchronize(), where);
    f->hf = true;
    f->hfBlock = frames_per_block;
    f->hfFrameRate = (float)frame_rate;
    f->hfRealtime = realtime_activity_labels != 0;
    return HW_OK;
}

int hw_fused_use_graphs(hw_fused* f, int32_t enable)
{
    if (!f) return Fail(HW_ERR_INVALID_ARG, "NULL engine");
    f->graphs = enable != 0;
    return HW_OK;
}

int hw_fused_set_tuning(hw_fused* f, const hw_fused_tuning* t, uint32_t n)
{
    if (!f || (n && !t)) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    for (uint32_t i = 0; i < n; ++i)
    {
        const uint32_t lpc = t[i].labeler_lanes_per_cta;
        if (lpc != 1 && lpc != 2 && lpc != 4) return Fail(HW_ERR_INVALID_ARG, "labeler_lanes_per_cta must be 1, 2 or 4");
        if (t[i].fuse_label_pulses > 1) return Fail(HW_ERR_INVALID_ARG, "fuse_label_pulses must be 0 or 1");
    }
    for (uint32_t i = 0; i < n; ++i)
        f->tuning[t[i].frames_per_chunk] = {t[i].fuse_label_pulses, t[i].labeler_lanes_per_cta};
    return HW_OK;
}

int hw_chunk_fused(hw_fused* f, hw_pool_chunk* table, uint32_t n_pools, void* stream)
{
    const hwk::NvtxRange range("hw_chunk_fused");
    if (!f || !table) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    if (n_pools != f->pools.size()) return Fail(HW_ERR_INVALID_ARG, "the table must list every pool of the engine");
    for (uint32_t p = 0; p < n_pools; ++p)
    {
        const hw_pool_chunk& c = table[p];
        if (!(c.d_trace || c.d_trace8) || !c.d_pulses || !c.d_lens || !c.d_overflows || (f->hf && !c.d_metrics))
            return Fail(HW_ERR_INVALID_ARG, "NULL buffer in the pool table");
        if (c.first_frame != f->pools[p].nextFrame) return Fail(HW_ERR_FRAME_ORDER, "Bad frame ID.");
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int b = (int)(f->step & 1);
    int rc;
    // the step that last used buffer b must be done before its tables are rewritten
    if ((rc = Collect(f, b))) return rc;
    if (f->sticky) return Fail(f->sticky, kDeferredMsg);
    int32_t counts[kNumLists];
    int maxFList[kNumLists];
    if ((rc = f->Schedule(table, b, counts, maxFList))) return rc;
    if ((uint32_t)counts[L_DME] > f->dmeCap)
    {
        // grow the DME scratch (graphs hold the old pointer)
        for (auto& g : f->graphCache) cudaGraphExecDestroy(g.second);
        f->graphCache.clear();
        HWF_CUDA(cudaFree(f->dmeScratch), "hw_chunk_fused");
        f->dmeScratch = nullptr;
        f->dmeCap = 0;
        if ((rc = Alloc(&f->dmeScratch, (size_t)counts[L_DME] * 3 * (kBins + 1) * kLane, "hw_chunk_fused"))) return rc;
        f->dmeCap = (uint32_t)counts[L_DME];
    }
    {
        TableCopy t{};
        uint64_t words = sizeof(PoolStep) / 4 * (uint64_t)n_pools;
        t.src[0] = reinterpret_cast<const uint32_t*>(f->mSteps[b]);
        t.dst[0] = reinterpret_cast<uint32_t*>(f->dSteps);
        t.words[0] = (uint32_t)words;
        t.n = 1;
        for (int l = 0; l < kNumLists; ++l)
            if (counts[l])
            {
                t.src[t.n] = reinterpret_cast<const uint32_t*>(f->mLists[b] + (size_t)l * f->lanes);
                t.dst[t.n] = reinterpret_cast<uint32_t*>(f->dLists + (size_t)l * f->lanes);
                t.words[t.n] = (uint32_t)counts[l];
                words += (uint64_t)counts[l];
                ++t.n;
            }
        const int blocks = (int)std::min<uint64_t>(148 * 4, (words + 255) / 256);
        TableCopyKernel<<<blocks, 256, 0, s>>>(t);
        HWF_CUDA(cudaGetLastError(), "hw_chunk_fused: step tables");
    }
    uint32_t launches = 0, graphLaunches = 0;
    if (f->graphs && !f->profiling)
    {
        std::vector<int64_t> key;
        for (int l = 0; l < kNumLists; ++l)
        {
            key.push_back(counts[l]);
            key.push_back(maxFList[l]);
        }
        // the learned start's proposal launches cover the estimating pools'
        // lane ranges: a plan is also which pools those are
        if (f->net)
            for (int p : f->dmePools) key.push_back(-1 - (int64_t)p);
        auto it = f->graphCache.find(key);
        if (it == f->graphCache.end() && ++f->planSeen[key] >= 2)
        {
            // second sighting of this plan: capture it
            if (!f->capStream)
                HWF_CUDA(cudaStreamCreateWithFlags(&f->capStream, cudaStreamNonBlocking), "hw_chunk_fused: capture");
            HWF_CUDA(cudaStreamBeginCapture(f->capStream, cudaStreamCaptureModeThreadLocal), "hw_chunk_fused: capture");
            uint32_t n = 0;
            rc = f->Launch(f->capStream, counts, maxFList, &n);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(f->capStream, &g);
            if (rc) { if (g) cudaGraphDestroy(g); return rc; }
            HWF_CUDA(ce, "hw_chunk_fused: capture");
            cudaGraphExec_t ge = nullptr;
            const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
            cudaGraphDestroy(g);
            HWF_CUDA(ie, "hw_chunk_fused: graph instantiation");
            it = f->graphCache.emplace(key, ge).first;
        }
        if (it != f->graphCache.end())
        {
            HWF_CUDA(cudaGraphLaunch(it->second, s), "hw_chunk_fused: graph launch");
            graphLaunches = 1;
        }
    }
    if (!graphLaunches && (rc = f->Launch(s, counts, maxFList, &launches))) return rc;
    ErrorOutKernel<<<1, 32, 0, s>>>(f->err, f->mErr[b]);
    HWF_CUDA(cudaGetLastError(), "hw_chunk_fused: failure word");
    HWF_CUDA(cudaEventRecord(f->ev[b], s), "hw_chunk_fused");
    f->inFlight[b] = true;
    f->lastLaunches = launches + 2;     // + the table and failure-word kernels
    f->lastGraphLaunches = graphLaunches;
    ++f->step;
    return HW_OK;
}

int hw_fused_set_learned_init(hw_fused* f, hw_learned_init* net)
{
    if (!f) return Fail(HW_ERR_INVALID_ARG, "NULL engine");
    if (net && !f->lProp)
    {
        const int rc = Alloc(&f->lProp, (size_t)f->lanes * 15 * kLane, "hw_fused_set_learned_init");
        if (rc) return rc;
    }
    if (net != f->net)
    {
        for (auto& g : f->graphCache) cudaGraphExecDestroy(g.second);
        f->graphCache.clear();
        f->planSeen.clear();
    }
    f->net = net;
    return HW_OK;
}

int hw_fused_set_overlap(hw_fused* f, int32_t mode)
{
    if (!f || mode < 0 || mode > 2) return Fail(HW_ERR_INVALID_ARG, "hw_fused_set_overlap: mode must be 0, 1 or 2");
    f->overlapMode = mode;
    return HW_OK;
}

int hw_fused_finish(hw_fused* f, void* stream)
{
    if (!f) return Fail(HW_ERR_INVALID_ARG, "NULL engine");
    (void)stream;
    int rc;
    for (int i = 0; i < 2; ++i)
    {
        // oldest step first
        const int b = (int)((f->step + i) & 1);
        if ((rc = Collect(f, b))) return rc;
    }
    if (f->sticky) return Fail(f->sticky, kDeferredMsg);
    return HW_OK;
}

int hw_fused_models(const hw_fused* f, uint32_t pool, hw_lane_model* d_out, hw_frame_interval* fi, void* stream)
{
    if (!f || !d_out || pool >= f->pools.size()) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    const PoolRt& P = f->pools[pool];
    HWF_CUDA(cudaMemcpyAsync(d_out, f->models + P.lane0, sizeof(hw_lane_model) * P.lanes, cudaMemcpyDeviceToDevice,
                             reinterpret_cast<cudaStream_t>(stream)),
             "hw_fused_models");
    if (fi) *fi = P.modelFi;
    return HW_OK;
}

int hw_fused_last_diag(const hw_fused* f, uint32_t pool, hw_dme_diag* d_out, int32_t* valid, void* stream)
{
    if (!f || !d_out || pool >= f->pools.size()) return Fail(HW_ERR_INVALID_ARG, "bad argument");
    const PoolRt& P = f->pools[pool];
    if (valid) *valid = P.diagValid ? 1 : 0;
    if (!P.diagValid) return HW_OK;
    HWF_CUDA(cudaMemcpyAsync(d_out, f->diag + P.lane0, sizeof(hw_dme_diag) * P.lanes, cudaMemcpyDeviceToDevice,
                             reinterpret_cast<cudaStream_t>(stream)),
             "hw_fused_last_diag");
    return HW_OK;
}

int hw_fused_profile(hw_fused* f, int32_t enable)
{
    if (!f) return Fail(HW_ERR_INVALID_ARG, "NULL engine");
    f->profiling = enable != 0;
    return HW_OK;
}

int hw_fused_stage_times(hw_fused* f, double ms[HW_NUM_STAGES], uint32_t launches[HW_NUM_STAGES])
{
    if (!f || !ms || !launches) return Fail(HW_ERR_INVALID_ARG, "NULL argument");
    for (int i = 0; i < HW_NUM_STAGES; ++i) { ms[i] = 0.0; launches[i] = 0; }
    for (const auto& m : f->evMarks)
    {
        HWF_CUDA(cudaEventSynchronize(f->evPool[m.second + 1]), "hw_fused_stage_times");
        float t = 0.0f;
        HWF_CUDA(cudaEventElapsedTime(&t, f->evPool[m.second], f->evPool[m.second + 1]), "hw_fused_stage_times");
        ms[m.first] += t;
        launches[m.first] += 1;
    }
    f->evMarks.clear();
    f->evUsed = 0;
    return HW_OK;
}

int hw_fused_last_step(const hw_fused* f, uint32_t* launches, uint32_t* graph_launches)
{
    if (!f) return Fail(HW_ERR_INVALID_ARG, "NULL engine");
    if (launches) *launches = f->lastLaunches;
    if (graph_launches) *graph_launches = f->lastGraphLaunches;
    return HW_OK;
}

}   // extern "C"
