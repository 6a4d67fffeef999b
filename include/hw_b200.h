/*
 * hw_b200 — C ABI of the B200-native smrt-basecaller trace-analysis chain.
 *
 * The chain is: multi-scale morphological baseliner -> baseline statistics
 * aggregation -> edge-scrubbed trace histogram -> detection-model EM ->
 * ROI-gated 13-state subframe Viterbi frame labeler -> pulse accumulator.
 * Each stage sits behind one opaque handle that mirrors one of the
 * reference's per-pool filter objects (src/basecaller/basecaller/traceAnalysis):
 *
 *   hw_baseliner             <- Baseliner / HostMultiScaleBaseliner
 *                               (traceAnalysis/Baseliner.h:53-79)
 *   hw_blstats_aggregator    <- BaselineStatsAggregator
 *                               (traceAnalysis/BaselineStatsAggregator.h:45-104)
 *   hw_histogram             <- TraceHistogramAccumulator
 *                               (traceAnalysis/TraceHistogramAccumulator.h:52-155)
 *   hw_dme                   <- CoreDMEstimator / DmeEmHost
 *                               (traceAnalysis/CoreDMEstimator.h:151-162)
 *   hw_labeler               <- FrameLabeler / FrameLabelerHost
 *                               (traceAnalysis/FrameLabeler.h:67-74)
 *   hw_pulse_accumulator     <- PulseAccumulator / HostPulseAccumulator
 *                               (traceAnalysis/PulseAccumulator.h:68-74)
 *   hw_analyzer              <- BatchAnalyzer + DetectionModelEstimator
 *                               (analyzer/BatchAnalyzer.cpp:149-375,
 *                                traceAnalysis/DetectionModelEstimator.cpp:93-160)
 *
 * Conventions
 *   - Every function returns an hw_status (0 = HW_OK). No exceptions cross
 *     the ABI; hw_last_error_string() describes the last failure on the
 *     calling thread.
 *   - Pointers named d_* are device pointers; the caller owns them.  State
 *     that persists between chunks is owned by the handle, in device memory.
 *   - `stream` is a cudaStream_t passed as void* (NULL = default stream).
 *     Calls are asynchronous on that stream unless documented otherwise.
 *     A handle is not re-entrant: issue its calls from one thread, in
 *     chunk order (the reference analyzer is non-reentrant per pool too,
 *     analyzer/BatchAnalyzer.h:75-78).
 *   - Batch layout is the reference BatchData block-major layout
 *     (dataTypes/BatchData.h:78-355): data[lane][frame][zmw] with 64 ZMWs per
 *     lane.
 *   - The lane structs below reproduce the member order and sizes of the
 *     reference's lane SoA types so buffers can be exchanged unchanged.
 */
#ifndef HW_B200_H_
#define HW_B200_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HW_LANE_SIZE   64   /* common/MongoConstants.h laneSize */
#define HW_NUM_ANALOGS 4    /* common/MongoConstants.h numAnalogs */
#define HW_NUM_BINS    300  /* dataTypes/PoolHistogram.h:47 LaneHistogram::numBins */
#define HW_NUM_STATES  13   /* traceAnalysis/SubframeLabelManager.h numStates */
#define HW_AUTOCORR_LAG 4   /* common/AutocorrAccumState.h lag */

typedef enum hw_status {
    HW_OK = 0,
    HW_ERR_INVALID_ARG = 1,      /* bad pointer, size or configuration value */
    HW_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    HW_ERR_BAD_POOL = 3,         /* batch belongs to another pool */
    HW_ERR_FRAME_ORDER = 4,      /* batch is not the next chunk in time */
    HW_ERR_NOT_INITIALIZED = 5,  /* e.g. histogram used before its first Reset */
    HW_ERR_UNSUPPORTED = 6,      /* option of the reference not built here */
    HW_ERR_TIMEOUT = 7,          /* a bounded device wait gave up */
    HW_ERR_OUT_OF_MEMORY = 8,
    HW_ERR_NUMERIC = 9,          /* a reference assertion on the data failed
                                    (e.g. histogram bounds, DME sanity checks) */
    HW_ERR_INTERNAL = 10
} hw_status;

/* BasecallerBaselinerConfig::FilterTypes (dataTypes/configs/BasecallerBaselinerConfig.h) */
typedef enum hw_filter_type {
    HW_FILTER_MULTISCALE_LARGE = 0,
    HW_FILTER_MULTISCALE_MEDIUM = 1,
    HW_FILTER_MULTISCALE_SMALL = 2,
    HW_FILTER_TWOSCALE_LARGE = 3,
    HW_FILTER_TWOSCALE_MEDIUM = 4,
    HW_FILTER_TWOSCALE_SMALL = 5
} hw_filter_type;

/* BasecallerRoiConfig::RoiFilterType */
typedef enum hw_roi_filter { HW_ROI_DEFAULT = 0, HW_ROI_NOOP = 1 } hw_roi_filter;

/* BasecallerAlgorithmConfig::ModelEstimationMode */
typedef enum hw_estimation_mode {
    HW_FIXED_ESTIMATIONS = 0,
    HW_INITIAL_ESTIMATIONS = 1,   /* SingleEstimateBatchAnalyzer */
    HW_DYNAMIC_ESTIMATIONS = 2    /* DynamicEstimateBatchAnalyzer */
} hw_estimation_mode;

/* One analog's kinetics and amplitude (pa-common AuxData::AnalogMode fields used on the path). */
typedef struct hw_analog {
    char  base_label;             /* 'A','C','G','T' */
    float rel_amplitude;          /* relAmplitude */
    float excess_noise_cv;        /* excessNoiseCV */
    float pulse_width_s;          /* pulseWidth, seconds */
    float ipd_s;                  /* interPulseDistance, seconds */
    float pw2_slow_step_ratio;    /* pw2SlowStepRatio */
    float ipd2_slow_step_ratio;   /* ipd2SlowStepRatio */
} hw_analog;

/* All parameters of the path.  hw_config_default() fills reference defaults. */
typedef struct hw_config {
    /* AnalysisConfig / MovieInfo */
    double   frame_rate;                 /* frames per second */
    float    photoelectron_sensitivity;  /* e-/DN; baseliner and histogram scaler */
    float    ref_snr;                    /* SNR of an analog with relAmplitude 1 */
    float    shot_var_coeff;             /* CoreDMEstimator::Configuration::shotVarCoeff */
    int16_t  pedestal;
    hw_analog analogs[HW_NUM_ANALOGS];   /* brightest first, dimmest last */

    /* BasecallerBaselinerConfig */
    int32_t  filter_type;                /* hw_filter_type */
    float    mean_bias_adjust;
    float    sigma_bias_adjust;
    float    mean_ema_scale_strides;
    float    sigma_ema_scale_strides;
    float    jump_suppression;

    /* BasecallerTraceHistogramConfig */
    float    bin_size_coeff;
    float    bin_size_low_bound_coeff;
    uint32_t baseline_stat_min_frame_count;
    float    fallback_baseline_sigma;

    /* BasecallerDmeConfig */
    uint32_t num_frames_pre_accum_stats;
    uint32_t min_frames_for_estimate;
    float    analog_mix_fraction_threshold[2];
    float    scale_snr_conf_tol;
    uint32_t em_iteration_limit;
    float    gtest_stat_factor;          /* < 0 disables the G-test (default -1) */
    int32_t  iterate_to_limit;
    float    min_analog_snr_thresh0;
    float    min_analog_snr_thresh1;
    float    pulse_amp_regularization;
    uint32_t model_update_method;        /* 0, 1 (default) or 2 */
    float    snr_drop_thresh;
    float    success_confidence_thresh;
    float    confidence_half_life[2];

    /* BasecallerFrameLabelerConfig */
    float    viterbi_alpha;
    float    viterbi_beta;
    float    viterbi_gamma;
    int32_t  roi_filter_type;            /* hw_roi_filter */
    float    roi_upper_threshold;
    float    roi_lower_threshold;

    /* BasecallerPulseAccumConfig */
    uint32_t max_calls_per_zmw;
    double   xsp_amp_thresh;
    float    xsp_width_thresh;

    /* BasecallerAlgorithmConfig */
    int32_t  model_estimation_mode;      /* hw_estimation_mode */
    /* StaticDetModelConfig (used only with HW_FIXED_ESTIMATIONS) */
    float    static_baseline_mean;
    float    static_baseline_variance;
} hw_config;

/* ---- Lane structs (64 ZMWs each, structure-of-arrays) ------------------ */

/* common/StatAccumState.h StatAccumStateT<float,64> */
typedef struct hw_stat_accum_state {
    float offset[HW_LANE_SIZE];
    float moment0[HW_LANE_SIZE];
    float moment1[HW_LANE_SIZE];
    float moment2[HW_LANE_SIZE];
} hw_stat_accum_state;

/* common/AutocorrAccumState.h AutocorrAccumState */
typedef struct hw_autocorr_accum_state {
    hw_stat_accum_state basic_stats;
    float   moment2[HW_LANE_SIZE];
    float   fbuf[HW_AUTOCORR_LAG][HW_LANE_SIZE];
    float   bbuf[HW_AUTOCORR_LAG][HW_LANE_SIZE];
    uint8_t bidx[2][HW_LANE_SIZE];
} hw_autocorr_accum_state;

/* dataTypes/BaselinerStatAccumState.h BaselinerStatAccumState */
typedef struct hw_baseliner_stats {
    hw_autocorr_accum_state full_autocorr;
    int16_t trace_min[HW_LANE_SIZE];
    int16_t trace_max[HW_LANE_SIZE];
    hw_stat_accum_state baseline_stats;
    float   raw_baseline_sum[HW_LANE_SIZE];
    hw_stat_accum_state background_stats;
} hw_baseliner_stats;

/* dataTypes/LaneDetectionModel.h LaneAnalogMode<PBHalf,64>; IEEE binary16 bits */
typedef struct hw_lane_analog_mode {
    uint16_t means[HW_LANE_SIZE];
    uint16_t vars[HW_LANE_SIZE];
    uint16_t weights[HW_LANE_SIZE];
} hw_lane_analog_mode;

/* dataTypes/LaneDetectionModel.h LaneModelParameters<PBHalf,64> (2048 bytes) */
typedef struct hw_lane_model {
    hw_lane_analog_mode analogs[HW_NUM_ANALOGS];
    hw_lane_analog_mode baseline;
    uint16_t confidence[HW_LANE_SIZE];
} hw_lane_model;

/* dataTypes/PoolHistogram.h LaneHistogram<float, unsigned short> */
typedef struct hw_lane_histogram {
    float    low_bound[HW_LANE_SIZE];
    float    bin_size[HW_LANE_SIZE];
    uint16_t outlier_count_low[HW_LANE_SIZE];
    uint16_t outlier_count_high[HW_LANE_SIZE];
    uint16_t bin_count[HW_NUM_BINS][HW_LANE_SIZE];
} hw_lane_histogram;

/* traceAnalysis/TraceHistogramAccumulator.h:41 LaneHistBounds */
typedef struct hw_lane_hist_bounds {
    float upper_bounds[HW_LANE_SIZE];
    float lower_bounds[HW_LANE_SIZE];
} hw_lane_hist_bounds;

/* dataTypes/Pulse.h Pulse (20 bytes; signals in 0.1 DN fixed point) */
typedef struct hw_pulse {
    uint32_t start;
    uint16_t width;
    uint16_t mean_signal;
    uint16_t mid_signal;
    uint16_t max_signal;
    float    signal_m2;
    uint8_t  label;        /* Pulse::NucleotideLabel: A=0, C, G, T, N, NONE */
    uint8_t  is_reject;
    uint8_t  pad_[2];
} hw_pulse;

/* Per-ZMW DME diagnostics (traceAnalysis/MaxLikelihoodDiagnostics.h; the
 * reference computes these but does not export them). */
typedef struct hw_dme_diag {
    int32_t iter_count[HW_LANE_SIZE];   /* iteration of first convergence */
    int32_t converged[HW_LANE_SIZE];
    float   log_like[HW_LANE_SIZE];
    int32_t status[HW_LANE_SIZE];       /* CoreDMEstimator::ZmwStatus bits */
    float   confidence[HW_LANE_SIZE];   /* confidence of the fresh estimate */
    int32_t lane_iterations;            /* EM iterations the lane executed */
    int32_t pad_[15];
} hw_dme_diag;

/* IntInterval<int32_t>: [lower, upper); empty when lower == upper. */
typedef struct hw_frame_interval {
    int32_t lower;
    int32_t upper;
} hw_frame_interval;

/* ---- Library ------------------------------------------------------------ */

const char* hw_last_error_string(void);
const char* hw_version(void);

/* Reference defaults for every parameter (PB_CONFIG_PARAM defaults in
 * in dataTypes/configs) plus the analog set of the synthetic workloads. */
int hw_config_default(hw_config* cfg);

/* Configuration checks of the reference (ValidateConfig<> specialisations and
 * the Configure() asserts). */
int hw_config_validate(const hw_config* cfg);

/* Transition matrix of the subframe Viterbi in log space, dense [to][from]
 * with -inf where the sparse pattern has no entry
 * (traceAnalysis/SubframeScorer.cpp:36-223). Host-only, synchronous. */
int hw_transition_matrix(const hw_config* cfg, float out[HW_NUM_STATES][HW_NUM_STATES]);

/* ---- Baseliner (traceAnalysis/Baseliner.h:53-79) ------------------------- */
typedef struct hw_baseliner hw_baseliner;
int hw_baseliner_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes,
                        uint32_t frames_per_chunk, hw_baseliner** out);
int hw_baseliner_destroy(hw_baseliner* b);
/* MultiScaleBaseliner::StartupLatency (traceAnalysis/MultiScaleBaseliner.h:92-99) */
int hw_baseliner_startup_latency(const hw_baseliner* b, uint32_t* frames);
/* FilterBaseline: d_trace[lanes][F][64] int16 -> d_out (same shape) and one
 * hw_baseliner_stats per lane.  first_frame must continue the previous call. */
int hw_baseliner_process(hw_baseliner* b, const int16_t* d_trace, int32_t first_frame,
                         int16_t* d_out, hw_baseliner_stats* d_stats, void* stream);
/* The same for chunks in the uint8 encoding (PacketLayout UINT8,
 * DeviceMultiScaleBaseliner.cu:84-101): each value is widened to int16 before
 * any arithmetic, as BlockView::Extract does (BatchData.h:160-180). */
int hw_baseliner_process_u8(hw_baseliner* b, const uint8_t* d_trace, int32_t first_frame, int16_t* d_out,
                            hw_baseliner_stats* d_stats, void* stream);

/* ---- Baseline statistics aggregator (BaselineStatsAggregator.h:45-104) -- */
typedef struct hw_blstats_aggregator hw_blstats_aggregator;
int hw_blstats_aggregator_create(uint32_t pool_id, uint32_t lanes, hw_blstats_aggregator** out);
int hw_blstats_aggregator_destroy(hw_blstats_aggregator* a);
int hw_blstats_aggregator_add(hw_blstats_aggregator* a, const hw_baseliner_stats* d_stats,
                              hw_frame_interval fi, void* stream);
int hw_blstats_aggregator_get(const hw_blstats_aggregator* a, hw_baseliner_stats* d_out,
                              hw_frame_interval* fi, void* stream);
int hw_blstats_aggregator_reset(hw_blstats_aggregator* a, void* stream);

/* ---- Trace histogram (TraceHistogramAccumulator.h:96-154) -------------- */
typedef struct hw_histogram hw_histogram;
int hw_histogram_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, hw_histogram** out);
int hw_histogram_destroy(hw_histogram* h);
/* AddBatch: edge-frame scrubbing with the fp16 models, then binning. */
int hw_histogram_add_batch(hw_histogram* h, const int16_t* d_traces, uint32_t frames,
                           hw_frame_interval fi, const hw_lane_model* d_models, void* stream);
/* Reset(const BaselinerMetrics&): bounds from aggregated baseline stats. */
int hw_histogram_reset_from_stats(hw_histogram* h, const hw_baseliner_stats* d_stats, void* stream);
/* Reset(UnifiedCudaArray<LaneHistBounds>): explicit bounds. */
int hw_histogram_reset_from_bounds(hw_histogram* h, const hw_lane_hist_bounds* d_bounds, void* stream);
/* Histogram(): copy out one hw_lane_histogram per lane. */
int hw_histogram_get(const hw_histogram* h, hw_lane_histogram* d_out, hw_frame_interval* fi,
                     void* stream);

/* ---- Detection-model estimator (CoreDMEstimator.h:151-162, DmeEmHost) --- */
typedef struct hw_dme hw_dme;
int hw_dme_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, hw_dme** out);
int hw_dme_destroy(hw_dme* d);
/* InitDetectionModels (DmeEmHost.cpp:857-925). */
int hw_dme_init_models(hw_dme* d, const hw_baseliner_stats* d_stats, hw_lane_model* d_models,
                       void* stream);
/* Estimate (DmeEmHost.cpp:131-615): EM on the histograms, confidence-weighted
 * update of d_models in place.  model_fi is the models' frame interval,
 * hist_fi the histograms'.  d_diag (may be NULL) receives per-ZMW EM
 * diagnostics.  Synchronous: a failed reference assertion returns
 * HW_ERR_NUMERIC. */
int hw_dme_estimate(hw_dme* d, const hw_lane_histogram* d_hist, const hw_baseliner_stats* d_stats,
                    hw_frame_interval hist_fi, hw_frame_interval model_fi,
                    hw_lane_model* d_models, hw_dme_diag* d_diag, void* stream);

/* hw_dme_estimate from a learned EM start (no counterpart in the reference):
 * d_proposal [lanes][15][64] (fractions, means, variances of the baseline and
 * the four analogs, see hw_dme_em_fit) replaces the reference start for every
 * ZMW whose proposal log-likelihood is not lower than the reference start's;
 * everything else (lane-wide stopping rule, confidence, blend) is the
 * reference's.  Synchronous like hw_dme_estimate. */
int hw_dme_estimate_proposal(hw_dme* d, const hw_lane_histogram* d_hist, const hw_baseliner_stats* d_stats,
                             hw_frame_interval hist_fi, hw_frame_interval model_fi, hw_lane_model* d_models,
                             hw_dme_diag* d_diag, const float* d_proposal, void* stream);

/* Per-lane phase clock of the next estimates (no counterpart in the
 * reference): with profiling on, every hw_dme_estimate /
 * hw_dme_estimate_proposal records for each lane, in SM clock cycles of the
 * lane's first thread: [0] model evolution, preliminary estimate and EM
 * set-up, [1] the start choice of a proposal (the proposal's E-step, which
 * the first iteration reuses when the proposal is kept, and the reference
 * start's log-likelihood), [2] the E-steps with the lane-wide convergence
 * vote, [3] the M-steps, [4] the confidence, blend and export, [5] the
 * lane's EM iterations, [6] the whole lane, [7] the lane's ZMWs that kept
 * the reference start.  hw_dme_phase_cycles copies the
 * [lanes][8] int64 table to host memory (synchronous). */
int hw_dme_profile_phases(hw_dme* d, int enable);
int hw_dme_phase_cycles(const hw_dme* d, int64_t* host_out, void* stream);

/* DetectionModelHost <-> LaneDetectionModel<PBHalf> (DetectionModelHost.h:
 * constructor from a LaneDetectionModel, ExportTo; DetectionModelHost.cpp:
 * 47-60, 226-234, 277-285) with the estimator's own conversion code: the
 * float model the EM works on, d_params [lanes][16][64] = baseline weight,
 * mean, variance, each analog's weight, mean, variance, confidence, and the
 * fp16 lane model (variances clamped to half(65000) on export). */
int hw_detection_model_import(const hw_lane_model* d_models, uint32_t lanes, float* d_params, void* stream);
int hw_detection_model_export(const float* d_params, uint32_t lanes, hw_lane_model* d_models, void* stream);
/* EvolveConfidence (DetectionModelHost.h:189-201): the confidence row of
 * d_params decays by exp2(-|center(to) - center(from)| / half_life). */
int hw_detection_model_evolve_confidence(float* d_params, uint32_t lanes, hw_frame_interval from,
                                         hw_frame_interval to, float half_life, void* stream);

/* Same estimate as hw_dme_estimate for callers that cannot allocate device
 * memory: code that runs inside a custom allocator's callbacks (where a
 * cudaMalloc would re-enter the allocator), or a real-time pipeline whose
 * device memory is sized once at start-up.  No counterpart in the reference.
 *
 * It needs no handle: the EM scratch is a fixed file-scope device array of
 * about 28 MiB (128 lanes x 3 x 301 x 64 floats) that every GPU loading the
 * library holds until the process exits.
 *   - At most 128 lanes per call (HW_ERR_INVALID_ARG above that): split a
 *     larger pool into sub-ranges of at most 128 lanes.
 *   - Synchronous: it returns after the estimate finished on `stream`.
 *   - All calls on a device share the one scratch array and its error word,
 *     so calls must not overlap on the GPU: callers serialise them (one
 *     host thread, one stream, or their own lock).  Overlapping calls (two
 *     host threads, two streams, or processes sharing a context) overwrite
 *     each other's scratch and can clear each other's error word, which
 *     gives wrong models without an error.
 *   - The first call on each device looks up the array's device address
 *     (once per device, with that device current), so make it before any
 *     stream capture.  With CUDA's default lazy module loading the first use
 *     of the library's DME code on a device loads the module, and that load
 *     allocates the array: warm the library up once per device outside the
 *     no-allocation region (any hw_dme_* call, or a first
 *     hw_dme_estimate_noalloc call), or load with CUDA_MODULE_LOADING=EAGER.
 *   - The looked-up addresses are not valid after cudaDeviceReset. */
int hw_dme_estimate_noalloc(const hw_config* cfg, uint32_t lanes, const hw_lane_histogram* d_hist,
                            const hw_baseliner_stats* d_stats, hw_frame_interval hist_fi,
                            hw_frame_interval model_fi, hw_lane_model* d_models, hw_dme_diag* d_diag,
                            void* stream);

/* ---- EM fit of single ZMWs, for the learned initializer ------------------
 * No counterpart in the reference.  Runs the EM steps of hw_dme_estimate
 * (same arithmetic) for every ZMW on its own for exactly max_iter iterations,
 * with no lane-wide stopping rule and no final confidence blend, from
 *   HW_EM_START_PLAIN     the reference's own start (PrelimEstimate and
 *                         ScaleModelSnr of d_models, DmeEmHost.cpp:161-361),
 *   HW_EM_START_PROPOSAL  d_proposal,
 *   HW_EM_START_BETTER    d_proposal unless its log-likelihood is lower than
 *                         (or not comparable with) the plain start's, in which
 *                         case the plain start is used ("fell back").
 * Per-lane layouts (floats unless stated): d_proposal, d_target, d_params
 * [15][64] = mixture fractions, means and variances of the baseline and the
 * four analog modes; d_iters int32 [5][64] = first iteration that passes the
 * reference's convergence test (or -1), first iteration whose parameters are
 * within `tol` of d_target (relative, with floors 0.01 / 1 DN / 1 DN^2 under
 * fractions / means / variances; -1 if never, max_iter if only the final
 * parameters are), fell back (0/1), status bits, and the number of
 * iterations after which one update first changed the parameters by at most
 * `tol` (same relative measure; -1 if never); d_loglike [3][64] = log-
 * likelihood of the plain start, of the start used, and of the last
 * iteration.  d_params_at_stop [15][64] (may be NULL) receives the
 * parameters at the first iteration that passes the reference's convergence
 * test, the estimate the reference keeps when it stops there (NaN where no
 * iteration passes).  d_target may be NULL.  d_scratch holds
 * hw_dme_em_fit_scratch_bytes(lanes) bytes.  Asynchronous. */
typedef enum hw_em_start {
    HW_EM_START_PLAIN = 0,
    HW_EM_START_PROPOSAL = 1,
    HW_EM_START_BETTER = 2
} hw_em_start;
int hw_dme_em_fit_scratch_bytes(uint32_t lanes, uint64_t* bytes);
int hw_dme_em_fit(const hw_config* cfg, uint32_t lanes, const hw_lane_histogram* d_hist,
                  const hw_baseliner_stats* d_stats, hw_frame_interval hist_fi, hw_frame_interval model_fi,
                  const hw_lane_model* d_models, int start, const float* d_proposal, const float* d_target,
                  float tol, uint32_t max_iter, float* d_scratch, float* d_params, int32_t* d_iters,
                  float* d_loglike, float* d_params_at_stop, void* stream);

/* ---- Learned DME initializer (no counterpart in the reference) ----------
 * A 302 -> 256 -> 256 -> 19 MLP with BF16 weights and activations, FP32
 * accumulation and GELU (tanh form) that proposes each ZMW's EM start from
 * its trace histogram and baseline statistics; hw_dme_em_fit with
 * HW_EM_START_BETTER runs the EM from the proposal and falls back to the
 * reference start when the proposal's log-likelihood is lower.
 * Rows: features [n][304] (300 sqrt bin shares, baseline mean and variance
 * in bin units, 2 zero pads), raw targets and outputs [n][32] (19 used:
 * baseline mean, log variance, 4 analog means, 4 log analog variances, 5
 * mixture fractions, 4 excess-noise terms; means in bins above the
 * histogram's low bound, variances in squared bins).  Network outputs are
 * standardised by the output mean/scale of the normalisation block
 * [in mean 304][in scale 304][out mean 32][out scale 32]. */
typedef struct hw_learned_init hw_learned_init;
int hw_learned_init_create(uint32_t max_batch, uint64_t seed, hw_learned_init** out);
int hw_learned_init_destroy(hw_learned_init* h);
int hw_learned_init_param_count(uint32_t* count);
/* FP32 parameters (W1 [256][304], b1, W2 [256][256], b2, W3 [32][256], b3)
 * and the normalisation block, to or from host memory (either may be NULL). */
int hw_learned_init_get_params(const hw_learned_init* h, float* host_params, float* host_norm);
int hw_learned_init_set_params(hw_learned_init* h, const float* host_params, const float* host_norm);
int hw_learned_init_features(uint32_t lanes, const hw_lane_histogram* d_hist, const hw_baseliner_stats* d_stats,
                             float* d_features, void* stream);
/* Targets from fitted parameters d_params [lanes][15][64] (hw_dme_em_fit layout). */
int hw_learned_init_targets(const hw_config* cfg, uint32_t lanes, const float* d_params,
                            const hw_lane_histogram* d_hist, float* d_targets, void* stream);
/* Standardised outputs d_out [n][32] of n rows (any n): one fused launch of
 * 128-row tiles on the tensor cores (tcgen05, accumulators in tensor memory;
 * BF16 inputs and activations, FP32 accumulation).  Asynchronous. */
int hw_learned_init_forward(hw_learned_init* h, const float* d_features, uint32_t n, float* d_out, void* stream);
/* Synchronous: HW_ERR_TIMEOUT (and the flag cleared) when a forward pass
 * since the last call gave up a bounded tensor-core wait -- its rows were
 * written as NaN, which the learned start's fallback test rejects. */
int hw_learned_init_forward_status(hw_learned_init* h);
/* Features, forward pass and EM start of lanes * 64 ZMWs in one launch:
 * equal to hw_learned_init_features -> hw_learned_init_forward ->
 * hw_learned_init_proposal without the [n][304] and [n][32] intermediates.
 * Asynchronous (hw_learned_init_forward_status reports a timed-out wait). */
int hw_learned_init_propose(hw_learned_init* h, uint32_t lanes, const hw_lane_histogram* d_hist,
                            const hw_baseliner_stats* d_stats, float* d_proposal, void* stream);
/* EM start [lanes][15][64] from the outputs of lanes * 64 rows. */
int hw_learned_init_proposal(const hw_learned_init* h, uint32_t lanes, const float* d_out,
                             const hw_lane_histogram* d_hist, float* d_proposal, void* stream);
/* Mean-squared-error gradients of n <= max_batch rows (rows d_index[i] when
 * d_index is not NULL); synchronous, *loss receives the loss. */
int hw_learned_init_gradients(hw_learned_init* h, const float* d_features, const float* d_targets,
                              const int32_t* d_index, uint32_t n, float* d_grad, float* loss, void* stream);
/* One AdamW step (betas 0.9/0.999, eps 1e-8, decay on weight matrices). */
int hw_learned_init_train_step(hw_learned_init* h, const float* d_features, const float* d_targets,
                               const int32_t* d_index, uint32_t n, float lr, float weight_decay, float* loss,
                               void* stream);

/* ---- Frame labeler (FrameLabeler.h:67-74, FrameLabelerHost.cpp:314-612) - */
typedef struct hw_labeler hw_labeler;
int hw_labeler_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes,
                      uint32_t frames_per_chunk, hw_labeler** out);
int hw_labeler_destroy(hw_labeler* l);
/* Labels lag the traces by hw_labeler_latent_frames() (24) frames.
 * d_labels[lanes][F][64] int16; d_latent_out[lanes][24][64] receives the
 * traces the first 24 labels belong to (LabelsBatch::LatentTrace);
 * d_viterbi_score[lanes][64] the anchor log-likelihood.
 * d_margin_or_null[lanes][F][64] float, if not NULL, receives the best path's
 * decision margin of every label: for label f < F - 1, the gap between the
 * winning and the best other candidate of the path state's row in the
 * Viterbi step of frame f + 1 (which chose label f; 0 on a tie, +inf when
 * only one candidate is finite); for the last label, the gap between the
 * largest and the next back-propagated end-state probability (the anchor
 * choice, FrameLabelerHost.cpp:410-418).  The first call with a margin
 * buffer allocates the handle's gap scratch (13 floats per frame and ZMW). */
int hw_labeler_process(hw_labeler* l, const int16_t* d_traces, const hw_lane_model* d_models,
                       int16_t* d_labels, int16_t* d_latent_out, float* d_viterbi_score,
                       float* d_margin_or_null, void* stream);
uint32_t hw_labeler_latent_frames(void);

/* ---- Pulse accumulator (PulseAccumulator.h:68-74, HostPulseAccumulator) - */
typedef struct hw_pulse_accumulator hw_pulse_accumulator;
int hw_pulse_accumulator_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes,
                                uint32_t frames_per_chunk, hw_pulse_accumulator** out);
int hw_pulse_accumulator_destroy(hw_pulse_accumulator* p);
/* d_pulses[lanes][64][max_calls_per_zmw]; d_lens/d_overflows[lanes][64];
 * d_blstats one hw_stat_accum_state per lane (PulseDetectorMetrics).
 * first_frame is the frame of d_labels[0]: the trace chunk's first frame
 * minus hw_labeler_latent_frames(), as in the reference's labels batch
 * metadata (LabelsBatch.h:112-121).  Pulse starts are first_frame + the
 * relative frame, in uint32 arithmetic. */
int hw_pulse_accumulator_process(hw_pulse_accumulator* p, const int16_t* d_labels,
                                 const int16_t* d_latent_trace, const int16_t* d_trace,
                                 int32_t first_frame, const hw_lane_model* d_models,
                                 hw_pulse* d_pulses, uint32_t* d_lens, uint32_t* d_overflows,
                                 hw_stat_accum_state* d_blstats, void* stream);

/* ---- Batch analyzer (analyzer/BatchAnalyzer.cpp:149-375) ----------------
 * One pool's complete chain: baseliner, the DetectionModelEstimator state
 * machine (DetectionModelEstimator.cpp:93-160: stats aggregation, histogram,
 * model initialisation and EM estimation), frame labeler and pulse
 * accumulator, with the SingleEstimate (HW_INITIAL_ESTIMATIONS) or
 * DynamicEstimate (HW_DYNAMIC_ESTIMATIONS) schedule of the reference.
 * max_pool_id is unused by the reference schedule and kept for symmetry. */
typedef struct hw_analyzer hw_analyzer;
int hw_analyzer_create(const hw_config* cfg, uint32_t pool_id, uint32_t lanes, uint32_t frames_per_chunk,
                       hw_analyzer** out);
int hw_analyzer_destroy(hw_analyzer* a);
/* Makes an analyzer start every estimate from the network's proposal
 * (hw_dme_estimate_proposal); NULL restores the reference start.  The network
 * is not owned and must outlive its use. */
int hw_analyzer_set_learned_init(hw_analyzer* a, hw_learned_init* net);

/* Checkpoints (the reference keeps pool state in stashable device
 * allocations, analyzer/BatchAnalyzer.cpp:80; this saves and restores it to
 * host memory).  The blob holds every buffer that carries state between
 * chunks (filter windows, statistics, histogram, detection models, labeler
 * latency state, open pulse segments) and the estimation schedule; an
 * analyzer created with the same configuration, pool, lanes and chunk
 * length continues exactly where the exporting one stopped.  Export and
 * import are synchronous on `stream`. */
int hw_analyzer_state_size(const hw_analyzer* a, uint64_t* bytes);
int hw_analyzer_state_export(const hw_analyzer* a, void* host_blob, uint64_t bytes, void* stream);
int hw_analyzer_state_import(hw_analyzer* a, const void* host_blob, uint64_t bytes, void* stream);

/* ---- HF metrics (HFMetricsFilter) -------------------------------------------
 * Replaces HFMetricsFilterHost / HFMetricsFilterDevice
 * (traceAnalysis/HFMetricsFilter.h:43-105, HFMetricsFilterHost.cpp:40-121,
 * dataTypes/BasecallingMetricsAccumulator.cpp:40-504): per ZMW, pulse and
 * trace metrics accumulated over blocks of frames_per_block frames and
 * emitted once a block is complete.
 *
 * hw_basecalling_metrics has the layout of Data::BasecallingMetrics
 * (dataTypes/BasecallingMetrics.h:47-86, 137 bytes per ZMW). */
typedef struct hw_basecalling_metrics {
    uint8_t  activity_label[HW_LANE_SIZE];          /* HQRFPhysicalStates: 0 EMPTY, 1 SINGLE, 2 MULTI, 3 LOW */
    uint16_t num_pulse_frames[HW_LANE_SIZE];
    uint16_t num_base_frames[HW_LANE_SIZE];
    uint16_t num_sandwiches[HW_LANE_SIZE];
    uint16_t num_half_sandwiches[HW_LANE_SIZE];
    uint16_t num_pulse_label_stutters[HW_LANE_SIZE];
    uint16_t num_bases[HW_LANE_SIZE];
    uint16_t num_pulses[HW_LANE_SIZE];
    float    pk_mid_signal[HW_NUM_ANALOGS][HW_LANE_SIZE];
    float    bp_zvar[HW_NUM_ANALOGS][HW_LANE_SIZE];
    float    pk_zvar[HW_NUM_ANALOGS][HW_LANE_SIZE];
    float    pk_max[HW_NUM_ANALOGS][HW_LANE_SIZE];
    uint16_t num_pk_mid_frames[HW_NUM_ANALOGS][HW_LANE_SIZE];
    uint16_t num_pk_mid_bases_by_analog[HW_NUM_ANALOGS][HW_LANE_SIZE];
    uint16_t num_bases_by_analog[HW_NUM_ANALOGS][HW_LANE_SIZE];
    uint16_t num_pulses_by_analog[HW_NUM_ANALOGS][HW_LANE_SIZE];
    float    frame_baseline_dws[HW_LANE_SIZE];
    float    frame_baseline_variance_dws[HW_LANE_SIZE];
    uint16_t num_frames_baseline[HW_LANE_SIZE];
    uint32_t start_frame[HW_LANE_SIZE];
    uint16_t num_frames[HW_LANE_SIZE];
    float    autocorrelation[HW_LANE_SIZE];
    float    pulse_detection_score[HW_LANE_SIZE];
    int16_t  pixel_checksum[HW_LANE_SIZE];
} hw_basecalling_metrics;

typedef struct hw_hfmetrics hw_hfmetrics;
/* HFMetricsFilter::Configure(sandwichTolerance, framesPerHFMetricBlock,
 * frameRate, realtimeActivityLabels) + a filter for one pool of `lanes`
 * lanes.  Activity labels need the trained classifier (hw_hfmetrics_set_cart);
 * until one is set they stay EMPTY, as with realtimeActivityLabels false. */
int hw_hfmetrics_create(uint32_t lanes, uint32_t frames_per_block, double frame_rate,
                        int32_t realtime_activity_labels, hw_hfmetrics** out);
int hw_hfmetrics_destroy(hw_hfmetrics* h);
/* The activity labeler's trained CART (ActivityLabeler::TrainedCart,
 * dataTypes/TrainedCartParams.h:44-53): n_nodes nodes (children, feature
 * index -- negative at a leaf --, threshold, leaf value), the half-sandwich
 * rate curve (2 coefficients, highest degree first) and its cap.  Host
 * arrays; copied. */
int hw_hfmetrics_set_cart(hw_hfmetrics* h, const int16_t* children_left, const int16_t* children_right,
                          const int8_t* feature, const float* threshold, const int8_t* value, uint32_t n_nodes,
                          const float hsw_curve[2], float max_acceptable_halfsandwich_rate);
/* HFMetricsFilter::operator() for one pulse batch of the pool: pulses
 * [lanes][64][max_calls] with counts d_lens [lanes][64]; the chunk's
 * baseliner metrics, models, frame-labeler Viterbi scores [lanes][64] and
 * pulse-detector baseline statistics [lanes]; first_frame and frames of the
 * pulse batch.  When the batch completes a block (last frame % block <
 * frames), the block's metrics go to d_out[lanes] and *emitted = 1; otherwise
 * d_out is untouched and *emitted = 0. */
int hw_hfmetrics_process(hw_hfmetrics* h, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                         const hw_baseliner_stats* d_baseliner_stats, const hw_lane_model* d_models,
                         const float* d_viterbi_score, const hw_stat_accum_state* d_pd_baseline_stats,
                         int32_t first_frame, uint32_t frames, hw_basecalling_metrics* d_out, int32_t* emitted,
                         void* stream);

/* ---- Ingest repacking (BlockRepacker) ---------------------------------------
 * Replaces the data shuffle of BlockRepacker
 * (appModules/BlockRepacker.cpp:200-345, BatchFiller::Process): sensor
 * packets -- num_blocks blocks of block_width ZMWs, each block stored
 * [num_frames][block_width] -- are gathered into the pools' TraceBatch
 * chunks [lanes][frames_per_chunk][64].  Pools cover ZMWs [0, num_zmw) in
 * order, lanes_per_pool lanes each (the last pool may have fewer).  One call
 * handles the packets of one chunk of frames; each packet's frames lie inside
 * that chunk and its block width is a multiple of 32 ZMWs (int16) or 64 ZMWs
 * (uint8), the reference's cache-line granularity. */
typedef struct hw_sensor_packet {
    uint64_t data_offset;       /* bytes from d_packet_data to the packet's first block */
    uint32_t start_zmw;
    int32_t  start_frame;
    uint32_t num_frames;
    uint32_t block_width;       /* ZMWs per block */
    uint32_t num_blocks;
    uint32_t reserved;
} hw_sensor_packet;

typedef struct hw_repacker hw_repacker;
/* encoding: 0 = int16, 1 = uint8 (PacketLayout::INT16 / UINT8). */
int hw_repacker_create(uint32_t num_zmw, uint32_t lanes_per_pool, uint32_t frames_per_chunk, int32_t encoding,
                       hw_repacker** out);
int hw_repacker_destroy(hw_repacker* r);
int hw_repacker_num_pools(const hw_repacker* r, uint32_t* n_pools);
/* Gathers the packets (host descriptors, data in device memory) into the
 * pools' chunks of frames [chunk_first_frame, chunk_first_frame +
 * frames_per_chunk): d_pool_chunks[n_pools] are device pointers.  Packets
 * must lie in the chunk and in [0, num_zmw); every covered element is
 * written, others are left unchanged. */
int hw_repack_chunk(hw_repacker* r, const hw_sensor_packet* packets, uint32_t n_packets, const void* d_packet_data,
                    int32_t chunk_first_frame, void* const* d_pool_chunks, void* stream);

/* ---- BAZ pulse encoding (bazio/encoding) ------------------------------------
 * Replaces the pulse serialization of the BAZ writer path
 * (PrelimHQFilter.cpp:63-120 + PacketBuffer::AddZmw, bazio/writing/PacketBuffer.h:143-210,
 * with the field machinery of bazio/encoding/ObjectToBaz.h,
 * FieldTransforms.h and FieldSerializers.h): each ZMW's pulses of a chunk
 * become a byte string, appended per ZMW.  A pulse encoding is a list of
 * fields; consecutive fields are packed little-endian into groups of at most
 * 64 bits, a new group starting when the current one is a whole number of
 * bytes or the next field would not fit (ObjectToBaz.h:373-393), and each
 * group's overflow bytes follow its main bytes in field order. */
enum {
    HW_BAZ_LABEL = 0, HW_BAZ_START_FRAME = 1, HW_BAZ_PULSE_WIDTH = 2, HW_BAZ_IS_BASE = 3,
    HW_BAZ_PKMAX = 4, HW_BAZ_PKMID = 5, HW_BAZ_PKMEAN = 6, HW_BAZ_PKVAR = 7
};
enum { HW_BAZ_NOOP = 0, HW_BAZ_DELTA = 1, HW_BAZ_FLOAT_FIXED = 2 };                 /* transforms */
enum { HW_BAZ_TRUNCATE = 0, HW_BAZ_SIMPLE_OVERFLOW = 1, HW_BAZ_COMPACT_OVERFLOW = 2 }; /* serializers */
typedef struct hw_baz_field {
    int32_t name;             /* HW_BAZ_LABEL ... HW_BAZ_PKVAR */
    int32_t store_signed;
    int32_t transform;        /* HW_BAZ_NOOP, HW_BAZ_DELTA, HW_BAZ_FLOAT_FIXED */
    int32_t scale;            /* FloatFixedCodec FixedPointScale */
    int32_t transform_bytes;  /* FloatFixedCodec NumBytes */
    int32_t serialize;        /* HW_BAZ_TRUNCATE, HW_BAZ_SIMPLE_OVERFLOW, HW_BAZ_COMPACT_OVERFLOW */
    int32_t num_bits;         /* main-portion bits (1..30) */
    int32_t overflow_bytes;   /* SimpleOverflow NumBytes */
} hw_baz_field;

/* The basecaller's two encodings (basecaller/dataTypes/PulseGroups.h:42-96):
 * 0 = ProductionPulses (3 fields, 2 nominal bytes, rejected pulses left
 * out), 1 = InternalPulses (8 fields, 6 nominal bytes, every pulse). */
int hw_baz_preset(int32_t which, hw_baz_field* fields, uint32_t* n_fields, int32_t* skip_rejects);

typedef struct hw_baz_encoder hw_baz_encoder;
/* An encoder for num_zmw ZMWs; the start-frame delta state of each ZMW is
 * kept across calls (the per-ZMW serializers of PrelimHQFilter). */
int hw_baz_encoder_create(const hw_baz_field* fields, uint32_t n_fields, int32_t skip_rejects, uint32_t num_zmw,
                          hw_baz_encoder** out);
int hw_baz_encoder_destroy(hw_baz_encoder* e);
/* Encode only ZMW 0, stride, 2 x stride, ... of every lane (PrelimHQConfig
 * zmwOutputStride, PrelimHQFilter.cpp:107-118); the others get empty byte
 * ranges and keep their state.  stride divides 64 (default 1). */
int hw_baz_encoder_set_zmw_stride(hw_baz_encoder* e, uint32_t stride);
/* The bound on a tile's look-back: after `polls` reads of a predecessor's
 * word that is not ready (about 100 ns apart; default 4,194,304) the tile
 * gives up and the call returns HW_ERR_TIMEOUT with the delta state
 * unchanged.  withhold_tile >= 0 makes that tile never publish its count --
 * for tests of the bounded wait only; -1 for normal use. */
int hw_baz_encoder_set_wait_limit(hw_baz_encoder* e, uint32_t polls, int32_t withhold_tile);
/* Encodes one chunk: pulses [num_zmw][max_calls] with counts d_lens[num_zmw]
 * (counts above max_calls read as max_calls).
 * d_offsets[num_zmw + 1] receives each ZMW's byte range in d_bytes (capacity
 * bytes_capacity), d_events[num_zmw] (may be NULL) its pulses encoded (the
 * PacketBuffer event count); *total_bytes the chunk's bytes.  When the chunk needs
 * more than bytes_capacity (or d_bytes is NULL) the call returns
 * HW_ERR_OUT_OF_MEMORY with the offsets and *total_bytes set, the delta
 * state unchanged and the contents of d_bytes unspecified, so the same call
 * with a larger buffer encodes the chunk.  One launch (tiles of 128 ZMWs
 * placed by a decoupled look-back whose polls are bounded: HW_ERR_TIMEOUT if
 * one gives up); synchronises the stream once, to learn the total. */
int hw_baz_encode(hw_baz_encoder* e, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                  uint8_t* d_bytes, uint64_t bytes_capacity, uint64_t* d_offsets, uint32_t* d_events,
                  uint64_t* total_bytes, void* stream);
/* hw_baz_encode without the synchronisation: enqueues the chunk on the
 * stream and returns.  d_offsets[num_zmw] holds the chunk's bytes once the
 * stream reaches it; calls in a row are ordered on the stream and each one
 * continues the delta state of the last one that fit in its buffer.  After
 * synchronising, hw_baz_encode_result reports the last finished call as
 * hw_baz_encode would have (HW_OK, HW_ERR_OUT_OF_MEMORY, HW_ERR_TIMEOUT). */
int hw_baz_encode_async(hw_baz_encoder* e, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                        uint8_t* d_bytes, uint64_t bytes_capacity, uint64_t* d_offsets, uint32_t* d_events,
                        void* stream);
int hw_baz_encode_result(hw_baz_encoder* e, uint64_t* total_bytes);

/* ---- Pulse compaction (for the download of a chunk's results) --------------
 * The pulse accumulator's output keeps max_calls slots a ZMW (BatchVectors,
 * DT/BatchVectors.h); hw_pulses_compact packs the valid records ZMW after
 * ZMW: d_out[d_offsets[z] .. d_offsets[z + 1]) are ZMW z's min(d_lens[z],
 * max_calls) pulses, d_offsets[num_zmw] their total.  The total is also
 * left in one of two mapped host slots (*slot says which), readable with
 * hw_pulse_compactor_total once the stream has passed the call, so a caller
 * can size the copy of one call's records while the next call is queued. */
typedef struct hw_pulse_compactor hw_pulse_compactor;
int hw_pulse_compactor_create(uint32_t num_zmw, hw_pulse_compactor** out);
int hw_pulse_compactor_destroy(hw_pulse_compactor* h);
int hw_pulses_compact(hw_pulse_compactor* h, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                      hw_pulse* d_out, uint64_t* d_offsets, uint32_t* slot, void* stream);
int hw_pulse_compactor_total(const hw_pulse_compactor* h, uint32_t slot, uint64_t* total);

/* ---- Preliminary HQ stage (PrelimHQFilterBody + BazAggregator packets) ------
 * Replaces basecaller/appModules/PrelimHQFilter.cpp:63-230 with the packet
 * side of bazio/writing/BazAggregator.h (PacketBufferManager.cpp:43-176).
 * Each chunk's pulses are BAZ-encoded and kept on the device for the last
 * lookback_blocks metric blocks.  At each metric block's end (every
 * chunks_per_block chunks) the stage marks ZMWs HQ -- the reference's
 * placeholder rule (PrelimHQFilter.cpp:163-215: all ZMWs when enable_prehq is
 * 0; otherwise, from the lookback_blocks-th block on, every
 * round(1 / hq_throttle_fraction)-th ZMW still pre-HQ, in ZMW order), or the
 * caller's marks -- and produces the block's checkpoint (BazAggregator::
 * ProduceBazBuffer): no bytes for a pre-HQ ZMW, its bytes of the block for an
 * HQ ZMW, and for a ZMW marked HQ at this block every block of the window,
 * oldest first; older data is dropped.  With `metrics` set the stage also
 * runs the aggregator's metric side (bazio/writing/MetricBufferManager.h:
 * 70-357) on the HF metrics passed in; hw_prelim_hq_metrics reports each
 * checkpoint's metric blocks. */
typedef struct hw_prelim_hq_config {
    uint32_t chunks_per_block;      /* ceil(framesPerHFMetricBlock / frames per chunk) */
    uint32_t lookback_blocks;       /* PrelimHQConfig lookbackSize (>= 1) */
    int32_t  enable_prehq;          /* PrelimHQConfig enablePreHQ */
    float    hq_throttle_fraction;  /* PrelimHQConfig hqThrottleFraction */
    uint32_t zmw_stride;            /* PrelimHQConfig zmwOutputStride (divides 64) */
    uint32_t metrics;               /* 1: run the metric side; 0: keep only the activity labels */
} hw_prelim_hq_config;

/* A checkpoint: device buffers owned by the stage, valid until its next call. */
typedef struct hw_baz_checkpoint {
    const uint8_t*  d_bytes;        /* total_bytes, ZMW after ZMW */
    uint64_t        total_bytes;
    const uint64_t* d_offsets;      /* [num_zmw + 1] */
    const uint32_t* d_events;       /* [num_zmw] pulses in each ZMW's bytes */
    const uint8_t*  d_hq;           /* [num_zmw] 1: HQ after this block */
    uint32_t        num_hq;
    uint32_t        block;          /* the metric block (from 0) */
} hw_baz_checkpoint;

/* Reference defaults: 8 chunks (4096-frame metric blocks of 512-frame
 * chunks), lookback 10, preliminary HQ off, throttle 0.10, stride 1. */
int hw_prelim_hq_config_default(hw_prelim_hq_config* cfg);
typedef struct hw_prelim_hq hw_prelim_hq;
/* fields/n_fields/skip_rejects: the pulse encoding, as hw_baz_encoder_create. */
int hw_prelim_hq_create(const hw_baz_field* fields, uint32_t n_fields, int32_t skip_rejects, uint32_t num_zmw,
                        const hw_prelim_hq_config* cfg, hw_prelim_hq** out);
int hw_prelim_hq_destroy(hw_prelim_hq* h);
/* One chunk of pulses of all num_zmw ZMWs (as hw_baz_encode).  d_metrics:
 * the HF metrics of a block that ended with this chunk (ceil(num_zmw / 64)
 * lanes, NULL otherwise); each ZMW's most recent activity label is kept
 * (MetricBufferManager::GetRecentActivityLabel).  d_marks: NULL for the
 * placeholder rule, or per ZMW 1 = mark HQ at this block's end.  When the
 * chunk ends a metric block, *produced = 1 and *out describes the
 * checkpoint.  Synchronises the stream (once a chunk, twice more at a
 * block's end). */
int hw_prelim_hq_process(hw_prelim_hq* h, const hw_pulse* d_pulses, const uint32_t* d_lens, uint32_t max_calls,
                         const hw_basecalling_metrics* d_metrics, const uint8_t* d_marks, int32_t* produced,
                         hw_baz_checkpoint* out, void* stream);
/* BazAggregator::Flush: the HQ ZMWs' bytes of the chunks of the unfinished block. */
int hw_prelim_hq_flush(hw_prelim_hq* h, int32_t* produced, hw_baz_checkpoint* out, void* stream);
/* Each ZMW's most recent activity label (HQRFPhysicalStates; 4 before any). */
int hw_prelim_hq_activity(hw_prelim_hq* h, uint8_t* d_out, void* stream);

/* One metric block of one ZMW as the BAZ file takes it: Primary::
 * SpiderMetricBlock (bazio/MetricBlock.h:58-124, MetricBlock<float, 1>), its
 * fields in the same order.  Its count setters take uint16_t
 * (bazio/MetricBlock.h:153-310), so aggregated counts arrive modulo 65536;
 * num_baseline_frames keeps 32 bits.  pixel_checksum and dme_status are never
 * set on this path (0). */
typedef struct hw_spider_metric_block {
    uint32_t num_frames, num_pulses, pulse_width, base_width;
    uint32_t num_sandwiches, num_half_sandwiches, num_pulse_label_stutters;
    float    pulse_detection_score, trace_autocorr;
    int16_t  pixel_checksum;
    uint8_t  dme_status, activity_label;
    float    pkmid[HW_NUM_ANALOGS];               /* A, C, G, T */
    uint32_t num_pkmid_frames[HW_NUM_ANALOGS];
    float    pkmax[HW_NUM_ANALOGS];
    uint32_t num_bases[HW_NUM_ANALOGS];
    uint32_t num_pkmid_bases[HW_NUM_ANALOGS];
    float    bpzvar[HW_NUM_ANALOGS];
    float    pkzvar[HW_NUM_ANALOGS];
    float    baseline, baseline_sd;
    uint32_t num_baseline_frames;
} hw_spider_metric_block;

/* The metric side of a checkpoint: device buffers owned by the stage, valid
 * until its next call.  ZMW z's blocks are d_blocks[d_offsets[z] ..
 * d_offsets[z + 1]). */
typedef struct hw_metric_checkpoint {
    const hw_spider_metric_block* d_blocks;
    uint64_t        total_blocks;
    const uint64_t* d_offsets;      /* [num_zmw + 1] */
    uint32_t        block;          /* the metric block (from 0), as the checkpoint's */
    uint32_t        reserved;
} hw_metric_checkpoint;

/* The metric blocks of the checkpoint that the last hw_prelim_hq_process or
 * hw_prelim_hq_flush produced (BazAggregator::ProduceBazBuffer / Flush ->
 * MetricBufferManager::GetMetrics; the stage must have been created with
 * `metrics` set).  Preliminary HQ off (CompleteMetricsGroup,
 * PrelimHQFilter.cpp:232-290, MetricBufferManager.h:240-250): one block per
 * ZMW per metric block, CompleteMetrics<uint16_t, half> converted as it
 * arrives.  Preliminary HQ on (ProductionMetricsGroup): a pre-HQ ZMW's blocks
 * wait in the lookback window and the oldest are aggregated into its pre-HQ
 * block; a ZMW marked HQ emits its pre-HQ block and the window's blocks
 * aggregated by runs of equal activity label, the last run kept open; an HQ
 * ZMW emits an aggregate each time the label changes; the flush emits every
 * open aggregate with data.  The reference aggregates an HQ ZMW into the
 * open aggregate at its stale lookback index (MetricBufferManager.h:263) and
 * walks a newly-HQ ZMW's window reading each buffer at the index of the
 * buffer before it (:318); both read other ZMWs' entries, or memory never
 * written, once ZMWs below were marked HQ inside the window.  The stage
 * follows each ZMW's own entries and aggregate, which equals the reference
 * wherever those slips are no-ops. */
int hw_prelim_hq_metrics(const hw_prelim_hq* h, hw_metric_checkpoint* out);

/* ---- Pool sets: uneven pools --------------------------
 * No single reference counterpart: the reference runs one BatchAnalyzer per
 * pool.  A pool set owns n_pools pools of any lane counts and chunk lengths
 * (every chunk length a multiple of 16 frames, at most 1024).  Pools whose
 * estimation schedules coincide -- same chunk length and same stagger class
 * pool % ceil(MinFramesForEstimate / F) -- share one batched analyzer, so
 * each stage of a step is one launch per class (hw_pool_set_layout reports
 * how many classes), and every pool's results equal those of its own
 * analyzer.  Each step processes one chunk of every pool from one packed
 * device buffer of int16 traces: pool p's chunk [lanes_p][F_p][64] starts at
 * element in_offsets[p].  Step s covers frames [s * F_p, (s + 1) * F_p). */
typedef struct hw_pool_set hw_pool_set;
int hw_pool_set_create(const hw_config* cfg, uint32_t n_pools, const uint32_t* lanes,
                       const uint32_t* frames_per_chunk, hw_pool_set** out);
int hw_pool_set_destroy(hw_pool_set* s);
int hw_pool_set_layout(const hw_pool_set* s, uint64_t* in_offsets, uint64_t* total_elements,
                       uint32_t* n_launch_groups);
/* emitted / estimated: host arrays of n_pools flags (may be NULL). */
int hw_pool_set_process(hw_pool_set* s, const int16_t* d_packed, int32_t step, int32_t* emitted,
                        int32_t* estimated, void* stream);
/* Device pointers to pool p's outputs of the last step (stable across steps):
 * pulses [lanes_p][64][max_calls_per_zmw], lengths and overflows [lanes_p][64]. */
int hw_pool_set_outputs(const hw_pool_set* s, uint32_t pool, hw_pulse** d_pulses, uint32_t** d_lens,
                        uint32_t** d_overflows);

/* ---- Fused chunk engine (hw_chunk_fused) ------------------------------------
 * Replaces the per-pool BatchAnalyzer loop of the basecaller
 * (AN/BatchAnalyzer.cpp:119-375 run once per pool and chunk by the
 * basecaller's analysis threads, BC/appModules/Basecaller.h:246-250) with one
 * call per chunk step for all pools.  The engine owns the state of every
 * pool, packed lane after lane; each stage of a step (baseline filter,
 * statistics merge, histogram, model initialisation, DME, histogram reset,
 * labeler, pulse accumulator) is ONE launch over the list of lanes of all
 * pools that take it this step, whatever their lane counts and chunk lengths.
 * Each pool keeps hw_analyzer's schedule (estimation mode, stagger by
 * pool_id % chunksPerEstimate) and its results equal those of an
 * hw_analyzer(pool_ids[p], lanes[p], frames_per_chunk[p]).
 *
 * A step enqueues its work on `stream` without waiting for the device: a
 * failure that only the device detects (the reference's histogram-bounds and
 * DME sanity assertions) is returned by the second call after the failing
 * step, or by hw_fused_finish, and from then on by every call (the
 * reference throws and the analysis stops).  With graphs enabled, every
 * step plan (which lanes take which stage) seen twice is captured as a CUDA
 * graph and replayed from then on. */
typedef struct hw_fused hw_fused;

typedef struct hw_pool_chunk {
    const int16_t* d_trace;     /* [lanes][F][64] int16 chunk, or NULL when d_trace8 is set */
    const uint8_t* d_trace8;    /* [lanes][F][64] uint8 chunk, or NULL */
    hw_pulse* d_pulses;         /* [lanes][64][max_calls_per_zmw] */
    uint32_t* d_lens;           /* [lanes][64] */
    uint32_t* d_overflows;      /* [lanes][64] */
    hw_basecalling_metrics* d_metrics;  /* [lanes] HF metrics records (with hw_fused_enable_hf_metrics) */
    int32_t first_frame;        /* must be the pool's next frame (0, F, 2F, ...) */
    int32_t emitted;            /* out: 0 while the reference returns no pulses (start-up) */
    int32_t estimated;          /* out: 1 when this step ran a full DME estimate */
    int32_t metrics_emitted;    /* out: 1 when d_metrics holds a completed block */
} hw_pool_chunk;

/* Adds the HF metrics filter to every pool's step (HFMetricsFilter, called
 * by the analyzers after the pulse accumulator, AN/BatchAnalyzer.cpp:201,
 * 278, 368): one lane-list launch per step; each pool's block metrics go to
 * its table row's d_metrics when a pulse batch ends a block.  The CART
 * arrays may be NULL (no activity labels); see hw_hfmetrics_set_cart. */
int hw_fused_enable_hf_metrics(hw_fused* f, uint32_t frames_per_block, double frame_rate,
                               int32_t realtime_activity_labels, const int16_t* children_left,
                               const int16_t* children_right, const int8_t* feature, const float* threshold,
                               const int8_t* value, uint32_t n_nodes, const float* hsw_curve,
                               float max_acceptable_halfsandwich_rate);

/* Kernel choices for the pools of one chunk length (see hw_fused_set_tuning). */
typedef struct hw_fused_tuning {
    uint32_t frames_per_chunk;      /* pools with this chunk length */
    uint32_t fuse_label_pulses;     /* 1: labeler and pulse accumulator in one kernel */
    uint32_t labeler_lanes_per_cta; /* 1, 2 or 4 lanes per labeler block */
    uint32_t reserved;
} hw_fused_tuning;

/* pool_ids may be NULL (pool p gets id p).  Every chunk length must be a
 * multiple of 16 frames in [48, 1024]. */
int hw_fused_create(const hw_config* cfg, uint32_t n_pools, const uint32_t* pool_ids, const uint32_t* lanes,
                    const uint32_t* frames_per_chunk, hw_fused** out);
int hw_fused_destroy(hw_fused* f);
/* Processes one chunk of every pool: table[n_pools], in creation order. */
int hw_chunk_fused(hw_fused* f, hw_pool_chunk* table, uint32_t n_pools, void* stream);
/* How a step uses the engine's second stream (results are the same in every
 * mode): 0 one stream; 1 (default) in a step with an estimate, the DME and
 * histogram reset beside the labeling of the pools without one; 2 also the
 * statistics merge and histogram beside the labeling (measured on the chip
 * workload: 2% slower for a 16,384-lane engine, within 1% for 4096 lanes). */
int hw_fused_set_overlap(hw_fused* f, int32_t mode);
/* Starts every estimate of the engine's pools from net's proposal, as
 * hw_analyzer_set_learned_init does for one pool (per ZMW the proposal is
 * kept unless its log-likelihood is below the reference start's); NULL
 * restores the reference start.  net is not owned and must outlive the
 * steps that use it; engines on different streams may share one. */
int hw_fused_set_learned_init(hw_fused* f, hw_learned_init* net);
/* Waits for the enqueued steps and returns any failure they reported. */
int hw_fused_finish(hw_fused* f, void* stream);
int hw_fused_use_graphs(hw_fused* f, int32_t enable);
/* Replaces the kernel choices of the listed chunk lengths (others keep the
 * defaults: separate labeler and pulse kernels, 2 lanes per labeler block). */
int hw_fused_set_tuning(hw_fused* f, const hw_fused_tuning* tuning, uint32_t n);
/* Device copy of pool p's current models and their frame interval. */
int hw_fused_models(const hw_fused* f, uint32_t pool, hw_lane_model* d_out, hw_frame_interval* fi, void* stream);
/* Pool `pool`'s diagnostics of its latest estimate ([lanes] hw_dme_diag), as
 * hw_analyzer_last_diag; *valid = 0 (and nothing copied) before its first. */
int hw_fused_last_diag(const hw_fused* f, uint32_t pool, hw_dme_diag* d_out, int32_t* valid, void* stream);
/* Stage timers with the meaning of hw_analyzer_profile / _stage_times (the
 * HW_STAGE_* indices; a fused labeler + pulse kernel counts as the labeler).
 * While profiling, steps are launched kernel by kernel, not from graphs. */
int hw_fused_profile(hw_fused* f, int32_t enable);
int hw_fused_stage_times(hw_fused* f, double* ms, uint32_t* launches);
/* Kernel launches and graph replays of the last step (graph nodes are not
 * counted as launches). */
int hw_fused_last_step(const hw_fused* f, uint32_t* launches, uint32_t* graph_launches);
/* BatchAnalyzer::operator(): d_trace[lanes][F][64] must be the next chunk
 * (first_frame == previous first_frame + F, starting at 0); otherwise
 * HW_ERR_FRAME_ORDER.  Pulses go to d_pulses[lanes][64][max_calls_per_zmw]
 * with counts in d_lens / d_overflows; *emitted is set to 0 while the
 * reference would return an empty pulse batch (start-up), 1 otherwise.
 * *estimated is set to 1 when this chunk ran a full DME estimate. */
int hw_analyzer_process(hw_analyzer* a, const int16_t* d_trace, int32_t first_frame, hw_pulse* d_pulses,
                        uint32_t* d_lens, uint32_t* d_overflows, int32_t* emitted, int32_t* estimated,
                        void* stream);
/* hw_analyzer_process for chunks in the uint8 encoding (see
 * hw_baseliner_process_u8); an analyzer may receive either encoding. */
int hw_analyzer_process_u8(hw_analyzer* a, const uint8_t* d_trace, int32_t first_frame, hw_pulse* d_pulses,
                           uint32_t* d_lens, uint32_t* d_overflows, int32_t* emitted, int32_t* estimated,
                           void* stream);
/* Current detection models of the pool and their frame interval. */
int hw_analyzer_models(const hw_analyzer* a, hw_lane_model* d_out, hw_frame_interval* fi, void* stream);
/* The last chunk's BaselinerMetrics (per-chunk baseliner statistics),
 * FrameLabelerMetrics::viterbiScore [lanes][64] and
 * PulseDetectorMetrics::baselineStats [lanes] -- the inputs of the HF metrics
 * filter (hw_hfmetrics_process).  Valid after a chunk that ran the labeler;
 * any pointer may be NULL. */
int hw_analyzer_chunk_metrics(const hw_analyzer* a, hw_baseliner_stats* d_baseliner_stats, float* d_viterbi_score,
                              hw_stat_accum_state* d_pd_baseline_stats, void* stream);
/* Diagnostics of the most recent DME estimate (*valid = 0 if none yet). */
int hw_analyzer_last_diag(const hw_analyzer* a, hw_dme_diag* d_out, int32_t* valid, void* stream);

/* Stage timers (the AnalysisProfiler stages of TA/AnalysisProfiler.h:31-60):
 * while enabled, CUDA events bracket every stage the analyzer enqueues;
 * hw_analyzer_stage_times synchronises, returns the summed device time and
 * launch count per stage since the previous call, and clears them. */
enum {
    HW_STAGE_BASELINE = 0,
    HW_STAGE_AGGREGATE = 1,
    HW_STAGE_HISTOGRAM = 2,
    HW_STAGE_MODEL_INIT = 3,
    HW_STAGE_DME = 4,
    HW_STAGE_HIST_RESET = 5,
    HW_STAGE_LABELER = 6,
    HW_STAGE_PULSES = 7,
    HW_STAGE_METRICS = 8,       /* HF metrics (hw_chunk_fused only) */
    HW_NUM_STAGES = 9
};
int hw_analyzer_profile(hw_analyzer* a, int32_t enable);
int hw_analyzer_stage_times(hw_analyzer* a, double ms[HW_NUM_STAGES], uint32_t launches[HW_NUM_STAGES]);

/* ---- Synthetic traces ------------------------------------------------------
 * Device generator used by the benchmarks and tests in place of camera data
 * (a counter-based RNG: every chunk is reproducible from seed, ZMW index and
 * frame index). */
typedef struct hw_gen_params {
    uint64_t seed;
    float    baseline_mean;      /* DN */
    float    baseline_sigma;     /* DN */
    float    amplitudes[HW_NUM_ANALOGS];   /* DN, brightest first */
    float    amp_cv;             /* per-pulse amplitude CV */
    float    pulse_width_mean;   /* frames (geometric) */
    float    ipd_mean;           /* frames (geometric gap) */
    float    shot_coeff;         /* added variance per DN of pulse signal */
    float    gain_sigma;         /* per-ZMW lognormal gain on amplitudes */
    float    empty_fraction;     /* fraction of ZMWs without pulses */
    float    walk_sigma;         /* baseline random-walk step, DN per frame */
    float    amp_scale_sigma;    /* extra per-ZMW lognormal amplitude factor */
    float    rate_min, rate_max; /* per-ZMW pulse rate (pulses/frame) if rate_max > 0 */
    float    decay_fraction;     /* amplitude decay reached at decay_frames */
    int32_t  decay_frames;
    int32_t  step_frame;         /* baseline step start frame (< 0: none) */
    float    step_dn;
    float    step_fraction;      /* fraction of ZMWs with the step */
} hw_gen_params;

/* Defaults of workload 0 (small), 1 (chip), 2 (uneven pools) and 4 (streaming). */
int hw_gen_params_default(int workload, hw_gen_params* p);
typedef struct hw_trace_generator hw_trace_generator;
int hw_trace_generator_create(const hw_gen_params* p, uint32_t lanes, uint64_t zmw_offset,
                              hw_trace_generator** out);
int hw_trace_generator_destroy(hw_trace_generator* g);
/* Writes frames [first_frame, first_frame + frames) for all lanes; chunks
 * must be requested in order. */
int hw_trace_generator_next(hw_trace_generator* g, int16_t* d_out, int32_t first_frame, uint32_t frames,
                            void* stream);

#ifdef __cplusplus
}   /* extern "C" */
#endif

#endif  /* HW_B200_H_ */
