"""ctypes / numpy mirrors of the structs declared in include/hw_b200.h.

The numpy dtypes reproduce the byte layout of the C structs (checked against
``sizeof`` by the tests), so lane buffers move between numpy, torch and the
C ABI without conversion.
"""
import ctypes as C

import numpy as np

LANE = 64
NUM_ANALOGS = 4
NUM_BINS = 300
NUM_STATES = 13
LATENT_FRAMES = 24          # ViterbiStitchLookback + ROI lookForward + stitchFrames

HW_OK = 0
HW_ERR_OUT_OF_MEMORY = 8
STATUS_NAMES = {
    0: "HW_OK", 1: "HW_ERR_INVALID_ARG", 2: "HW_ERR_CUDA", 3: "HW_ERR_BAD_POOL",
    4: "HW_ERR_FRAME_ORDER", 5: "HW_ERR_NOT_INITIALIZED", 6: "HW_ERR_UNSUPPORTED",
    7: "HW_ERR_TIMEOUT", 8: "HW_ERR_OUT_OF_MEMORY", 9: "HW_ERR_NUMERIC",
    10: "HW_ERR_INTERNAL",
}

FILTER_TYPES = {
    "MultiScaleLarge": 0, "MultiScaleMedium": 1, "MultiScaleSmall": 2,
    "TwoScaleLarge": 3, "TwoScaleMedium": 4, "TwoScaleSmall": 5,
}
FIXED_ESTIMATIONS, INITIAL_ESTIMATIONS, DYNAMIC_ESTIMATIONS = 0, 1, 2
EM_START_PLAIN, EM_START_PROPOSAL, EM_START_BETTER = 0, 1, 2


class Analog(C.Structure):
    _fields_ = [
        ("base_label", C.c_char),
        ("rel_amplitude", C.c_float),
        ("excess_noise_cv", C.c_float),
        ("pulse_width_s", C.c_float),
        ("ipd_s", C.c_float),
        ("pw2_slow_step_ratio", C.c_float),
        ("ipd2_slow_step_ratio", C.c_float),
    ]


class Config(C.Structure):
    _fields_ = [
        ("frame_rate", C.c_double),
        ("photoelectron_sensitivity", C.c_float),
        ("ref_snr", C.c_float),
        ("shot_var_coeff", C.c_float),
        ("pedestal", C.c_int16),
        ("analogs", Analog * NUM_ANALOGS),
        ("filter_type", C.c_int32),
        ("mean_bias_adjust", C.c_float),
        ("sigma_bias_adjust", C.c_float),
        ("mean_ema_scale_strides", C.c_float),
        ("sigma_ema_scale_strides", C.c_float),
        ("jump_suppression", C.c_float),
        ("bin_size_coeff", C.c_float),
        ("bin_size_low_bound_coeff", C.c_float),
        ("baseline_stat_min_frame_count", C.c_uint32),
        ("fallback_baseline_sigma", C.c_float),
        ("num_frames_pre_accum_stats", C.c_uint32),
        ("min_frames_for_estimate", C.c_uint32),
        ("analog_mix_fraction_threshold", C.c_float * 2),
        ("scale_snr_conf_tol", C.c_float),
        ("em_iteration_limit", C.c_uint32),
        ("gtest_stat_factor", C.c_float),
        ("iterate_to_limit", C.c_int32),
        ("min_analog_snr_thresh0", C.c_float),
        ("min_analog_snr_thresh1", C.c_float),
        ("pulse_amp_regularization", C.c_float),
        ("model_update_method", C.c_uint32),
        ("snr_drop_thresh", C.c_float),
        ("success_confidence_thresh", C.c_float),
        ("confidence_half_life", C.c_float * 2),
        ("viterbi_alpha", C.c_float),
        ("viterbi_beta", C.c_float),
        ("viterbi_gamma", C.c_float),
        ("roi_filter_type", C.c_int32),
        ("roi_upper_threshold", C.c_float),
        ("roi_lower_threshold", C.c_float),
        ("max_calls_per_zmw", C.c_uint32),
        ("xsp_amp_thresh", C.c_double),
        ("xsp_width_thresh", C.c_float),
        ("model_estimation_mode", C.c_int32),
        ("static_baseline_mean", C.c_float),
        ("static_baseline_variance", C.c_float),
    ]

    def copy(self):
        c = Config()
        C.memmove(C.byref(c), C.byref(self), C.sizeof(Config))
        return c


class GenParams(C.Structure):
    _fields_ = [
        ("seed", C.c_uint64),
        ("baseline_mean", C.c_float),
        ("baseline_sigma", C.c_float),
        ("amplitudes", C.c_float * NUM_ANALOGS),
        ("amp_cv", C.c_float),
        ("pulse_width_mean", C.c_float),
        ("ipd_mean", C.c_float),
        ("shot_coeff", C.c_float),
        ("gain_sigma", C.c_float),
        ("empty_fraction", C.c_float),
        ("walk_sigma", C.c_float),
        ("amp_scale_sigma", C.c_float),
        ("rate_min", C.c_float),
        ("rate_max", C.c_float),
        ("decay_fraction", C.c_float),
        ("decay_frames", C.c_int32),
        ("step_frame", C.c_int32),
        ("step_dn", C.c_float),
        ("step_fraction", C.c_float),
    ]


class FrameInterval(C.Structure):
    _fields_ = [("lower", C.c_int32), ("upper", C.c_int32)]

    def __repr__(self):
        return f"[{self.lower}, {self.upper})"

    def tuple(self):
        return (self.lower, self.upper)


def _f32(n): return (np.float32, (n,))


STAT_ACCUM_DT = np.dtype([("offset", np.float32, (LANE,)), ("moment0", np.float32, (LANE,)),
                          ("moment1", np.float32, (LANE,)), ("moment2", np.float32, (LANE,))])
AUTOCORR_DT = np.dtype([("basic_stats", STAT_ACCUM_DT), ("moment2", np.float32, (LANE,)),
                        ("fbuf", np.float32, (4, LANE)), ("bbuf", np.float32, (4, LANE)),
                        ("bidx", np.uint8, (2, LANE))])
BLSTATS_DT = np.dtype([("full_autocorr", AUTOCORR_DT), ("trace_min", np.int16, (LANE,)),
                       ("trace_max", np.int16, (LANE,)), ("baseline_stats", STAT_ACCUM_DT),
                       ("raw_baseline_sum", np.float32, (LANE,)),
                       ("background_stats", STAT_ACCUM_DT)])
ANALOG_MODE_DT = np.dtype([("means", np.uint16, (LANE,)), ("vars", np.uint16, (LANE,)),
                           ("weights", np.uint16, (LANE,))])
LANE_MODEL_DT = np.dtype([("analogs", ANALOG_MODE_DT, (NUM_ANALOGS,)), ("baseline", ANALOG_MODE_DT),
                          ("confidence", np.uint16, (LANE,))])
LANE_HIST_DT = np.dtype([("low_bound", np.float32, (LANE,)), ("bin_size", np.float32, (LANE,)),
                         ("outlier_count_low", np.uint16, (LANE,)),
                         ("outlier_count_high", np.uint16, (LANE,)),
                         ("bin_count", np.uint16, (NUM_BINS, LANE))])
HIST_BOUNDS_DT = np.dtype([("upper_bounds", np.float32, (LANE,)), ("lower_bounds", np.float32, (LANE,))])
PULSE_DT = np.dtype([("start", np.uint32), ("width", np.uint16), ("mean_signal", np.uint16),
                     ("mid_signal", np.uint16), ("max_signal", np.uint16), ("signal_m2", np.float32),
                     ("label", np.uint8), ("is_reject", np.uint8), ("pad_", np.uint8, (2,))])
DME_DIAG_DT = np.dtype([("iter_count", np.int32, (LANE,)), ("converged", np.int32, (LANE,)),
                        ("log_like", np.float32, (LANE,)), ("status", np.int32, (LANE,)),
                        ("confidence", np.float32, (LANE,)), ("lane_iterations", np.int32),
                        ("pad_", np.int32, (15,))])

_L, _A = (LANE,), (NUM_ANALOGS, LANE)
BASECALLING_METRICS_DT = np.dtype([
    ("activity_label", np.uint8, _L), ("num_pulse_frames", np.uint16, _L), ("num_base_frames", np.uint16, _L),
    ("num_sandwiches", np.uint16, _L), ("num_half_sandwiches", np.uint16, _L),
    ("num_pulse_label_stutters", np.uint16, _L), ("num_bases", np.uint16, _L), ("num_pulses", np.uint16, _L),
    ("pk_mid_signal", np.float32, _A), ("bp_zvar", np.float32, _A), ("pk_zvar", np.float32, _A),
    ("pk_max", np.float32, _A), ("num_pk_mid_frames", np.uint16, _A), ("num_pk_mid_bases_by_analog", np.uint16, _A),
    ("num_bases_by_analog", np.uint16, _A), ("num_pulses_by_analog", np.uint16, _A),
    ("frame_baseline_dws", np.float32, _L), ("frame_baseline_variance_dws", np.float32, _L),
    ("num_frames_baseline", np.uint16, _L), ("start_frame", np.uint32, _L), ("num_frames", np.uint16, _L),
    ("autocorrelation", np.float32, _L), ("pulse_detection_score", np.float32, _L),
    ("pixel_checksum", np.int16, _L)])
HQRF_EMPTY, HQRF_SINGLE, HQRF_MULTI, HQRF_LOW = 0, 1, 2, 3

# hw_sensor_packet (repacker input descriptor)
SENSOR_PACKET_DT = np.dtype([("data_offset", np.uint64), ("start_zmw", np.uint32), ("start_frame", np.int32),
                             ("num_frames", np.uint32), ("block_width", np.uint32), ("num_blocks", np.uint32),
                             ("reserved", np.uint32)])

# hw_pool_chunk: one pool's row of the hw_chunk_fused table (device pointers as integers)
POOL_CHUNK_DT = np.dtype([("d_trace", np.uint64), ("d_trace8", np.uint64), ("d_pulses", np.uint64),
                          ("d_lens", np.uint64), ("d_overflows", np.uint64), ("d_metrics", np.uint64),
                          ("first_frame", np.int32), ("emitted", np.int32), ("estimated", np.int32),
                          ("metrics_emitted", np.int32)])
# hw_baz_field (one field of a BAZ pulse encoding)
BAZ_FIELD_DT = np.dtype([(n, np.int32) for n in ("name", "store_signed", "transform", "scale", "transform_bytes",
                                                  "serialize", "num_bits", "overflow_bytes")])
BAZ_LABEL, BAZ_START_FRAME, BAZ_PULSE_WIDTH, BAZ_IS_BASE, BAZ_PKMAX, BAZ_PKMID, BAZ_PKMEAN, BAZ_PKVAR = range(8)
BAZ_NOOP, BAZ_DELTA, BAZ_FLOAT_FIXED = range(3)
BAZ_TRUNCATE, BAZ_SIMPLE_OVERFLOW, BAZ_COMPACT_OVERFLOW = range(3)
BAZ_PRODUCTION, BAZ_INTERNAL = 0, 1

# hw_prelim_hq_config and hw_baz_checkpoint
PRELIM_HQ_CONFIG_DT = np.dtype([("chunks_per_block", np.uint32), ("lookback_blocks", np.uint32),
                                ("enable_prehq", np.int32), ("hq_throttle_fraction", np.float32),
                                ("zmw_stride", np.uint32), ("metrics", np.uint32)])
BAZ_CHECKPOINT_DT = np.dtype([("d_bytes", np.uint64), ("total_bytes", np.uint64), ("d_offsets", np.uint64),
                              ("d_events", np.uint64), ("d_hq", np.uint64), ("num_hq", np.uint32),
                              ("block", np.uint32)])

# hw_spider_metric_block (Primary::SpiderMetricBlock) and hw_metric_checkpoint
_N4 = (NUM_ANALOGS,)
SPIDER_METRIC_BLOCK_DT = np.dtype([
    ("num_frames", np.uint32), ("num_pulses", np.uint32), ("pulse_width", np.uint32), ("base_width", np.uint32),
    ("num_sandwiches", np.uint32), ("num_half_sandwiches", np.uint32), ("num_pulse_label_stutters", np.uint32),
    ("pulse_detection_score", np.float32), ("trace_autocorr", np.float32), ("pixel_checksum", np.int16),
    ("dme_status", np.uint8), ("activity_label", np.uint8), ("pkmid", np.float32, _N4),
    ("num_pkmid_frames", np.uint32, _N4), ("pkmax", np.float32, _N4), ("num_bases", np.uint32, _N4),
    ("num_pkmid_bases", np.uint32, _N4), ("bpzvar", np.float32, _N4), ("pkzvar", np.float32, _N4),
    ("baseline", np.float32), ("baseline_sd", np.float32), ("num_baseline_frames", np.uint32)])
METRIC_CHECKPOINT_DT = np.dtype([("d_blocks", np.uint64), ("total_blocks", np.uint64), ("d_offsets", np.uint64),
                                 ("block", np.uint32), ("reserved", np.uint32)])

FUSED_TUNING_DT = np.dtype([("frames_per_chunk", np.uint32), ("fuse_label_pulses", np.uint32),
                            ("labeler_lanes_per_cta", np.uint32), ("reserved", np.uint32)])

SIZES = {
    "hw_stat_accum_state": (STAT_ACCUM_DT, 1024),
    "hw_autocorr_accum_state": (AUTOCORR_DT, 3456),
    "hw_baseliner_stats": (BLSTATS_DT, 6016),
    "hw_lane_model": (LANE_MODEL_DT, 2048),
    "hw_lane_histogram": (LANE_HIST_DT, 39168),
    "hw_lane_hist_bounds": (HIST_BOUNDS_DT, 512),
    "hw_pulse": (PULSE_DT, 20),
    "hw_dme_diag": (DME_DIAG_DT, 1344),
    "hw_pool_chunk": (POOL_CHUNK_DT, 64),
    "hw_basecalling_metrics": (BASECALLING_METRICS_DT, 8768),
    "hw_sensor_packet": (SENSOR_PACKET_DT, 32),
    "hw_fused_tuning": (FUSED_TUNING_DT, 16),
    "hw_baz_field": (BAZ_FIELD_DT, 32),
    "hw_prelim_hq_config": (PRELIM_HQ_CONFIG_DT, 24),
    "hw_baz_checkpoint": (BAZ_CHECKPOINT_DT, 48),
    "hw_spider_metric_block": (SPIDER_METRIC_BLOCK_DT, 164),
    "hw_metric_checkpoint": (METRIC_CHECKPOINT_DT, 32),
}


def ptr(a):
    """ctypes void pointer to a numpy array's data (or None)."""
    if a is None:
        return None
    return C.c_void_p(a.ctypes.data)


def f16_to_f32(bits):
    return np.asarray(bits, dtype=np.uint16).view(np.float16).astype(np.float32)


def f32_to_f16(x):
    return np.asarray(x, dtype=np.float32).astype(np.float16).view(np.uint16)
