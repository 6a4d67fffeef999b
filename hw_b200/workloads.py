"""Pinned configurations of the synthetic workloads.

All workloads use the AnalysisConfig the synthetic traces are drawn from:
frame rate 100 fps, photoelectron sensitivity 1, pedestal 0, shot-noise
coefficient 0.5 (the generator adds 0.5 x signal to the baseline variance),
four analogs with relative amplitudes 4.0 / 2.5 / 1.6 / 1.0 (amplitudes
80 / 50 / 32 / 20 DN over a 200 DN baseline with sigma 8 DN), excess-noise CV
0.1, pulse width 0.08 s, inter-pulse distance 0.14 s.  refSnr, the SNR of the
relative-amplitude-1 analog, is therefore 20 / 8 = 2.5.

small_config() additionally shortens the start-up so that 8 chunks of 512
frames produce pulses (reference defaults need 9216 + 5120 frames before the
first estimate): TwoScaleMedium filter, SigmaEmaScaleStrides 8,
NumFramesPreAccumStats 512, MinFramesForEstimate 2048, single-estimate
analyzer.
"""
from . import abi

AMPLITUDES_DN = (80.0, 50.0, 32.0, 20.0)
BASELINE_DN = 200.0
BASELINE_SIGMA_DN = 8.0


def _base():
    cfg = abi.Config()
    cfg.frame_rate = 100.0
    cfg.photoelectron_sensitivity = 1.0
    cfg.ref_snr = AMPLITUDES_DN[3] / BASELINE_SIGMA_DN
    cfg.shot_var_coeff = 0.5
    cfg.pedestal = 0
    for i, (lbl, amp) in enumerate(zip(b"ACGT", AMPLITUDES_DN)):
        a = cfg.analogs[i]
        a.base_label = bytes([lbl])
        a.rel_amplitude = amp / AMPLITUDES_DN[3]
        a.excess_noise_cv = 0.1
        a.pulse_width_s = 0.08
        a.ipd_s = 0.14
        a.pw2_slow_step_ratio = 0.0
        a.ipd2_slow_step_ratio = 0.0
    # BasecallerBaselinerConfig defaults
    cfg.filter_type = abi.FILTER_TYPES["MultiScaleLarge"]
    cfg.mean_bias_adjust = 0.0
    cfg.sigma_bias_adjust = 0.0
    cfg.mean_ema_scale_strides = 0.0
    cfg.sigma_ema_scale_strides = 512.0
    cfg.jump_suppression = 0.0
    # BasecallerTraceHistogramConfig defaults
    cfg.bin_size_coeff = 0.2
    cfg.bin_size_low_bound_coeff = 1.0
    cfg.baseline_stat_min_frame_count = 50
    cfg.fallback_baseline_sigma = 10.0
    # BasecallerDmeConfig defaults
    cfg.num_frames_pre_accum_stats = 1000
    cfg.min_frames_for_estimate = 4000
    cfg.analog_mix_fraction_threshold[0] = 0.039 / 3
    cfg.analog_mix_fraction_threshold[1] = 0.039
    cfg.scale_snr_conf_tol = 1.0
    cfg.em_iteration_limit = 20
    cfg.gtest_stat_factor = -1.0
    cfg.iterate_to_limit = 0
    cfg.min_analog_snr_thresh0 = 2.0
    cfg.min_analog_snr_thresh1 = 4.0
    cfg.pulse_amp_regularization = 0.0
    cfg.model_update_method = 1
    cfg.snr_drop_thresh = 1.0
    cfg.success_confidence_thresh = 0.10
    cfg.confidence_half_life[0] = 4096.0
    cfg.confidence_half_life[1] = 12000.0
    # BasecallerFrameLabelerConfig defaults
    cfg.viterbi_alpha = 1.0
    cfg.viterbi_beta = 1.0
    cfg.viterbi_gamma = 1.0
    cfg.roi_filter_type = 0
    cfg.roi_upper_threshold = 7.0
    cfg.roi_lower_threshold = 2.0
    # BasecallerPulseAccumConfig defaults
    cfg.max_calls_per_zmw = 48
    cfg.xsp_amp_thresh = 0.70
    cfg.xsp_width_thresh = 3.5
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    cfg.static_baseline_mean = 0.0
    cfg.static_baseline_variance = 100.0
    return cfg


def chip_config():
    """Reference defaults (MultiScaleLarge, dynamic estimation) on the synthetic analogs."""
    return _base()


def small_config():
    """Shortened start-up so a 4096-frame run reaches labeling (see module doc)."""
    cfg = _base()
    cfg.filter_type = abi.FILTER_TYPES["TwoScaleMedium"]
    cfg.sigma_ema_scale_strides = 8.0
    cfg.num_frames_pre_accum_stats = 512
    cfg.min_frames_for_estimate = 2048
    cfg.model_estimation_mode = abi.INITIAL_ESTIMATIONS
    return cfg


def startup_chunks(cfg, pools, frames=512, latency=None):
    """Chunks of `frames` until every one of `pools` pools of the dynamic
    schedule has entered its periodic estimation cycle: the baseliner's
    start-up latency (`latency` frames, or the library's value for `cfg`),
    the stagger of the last pool, the statistics pre-accumulation and one
    estimation period."""
    if latency is None:
        import ctypes as C
        from . import native
        b = C.c_void_p()
        native.check(native.lib().hw_baseliner_create(C.byref(cfg), 0, 1, frames, C.byref(b)))
        lat = C.c_uint32()
        native.lib().hw_baseliner_startup_latency(b, C.byref(lat))
        native.lib().hw_baseliner_destroy(b)
        latency = lat.value
    chunks_per_est = (max(cfg.min_frames_for_estimate, 1) + frames - 1) // frames
    last_delay = ((pools - 1) % chunks_per_est) * frames
    start = (latency + last_delay + frames - 1) // frames            # first chunk the last pool analyses
    pre = (cfg.num_frames_pre_accum_stats + frames - 1) // frames    # histogram start-up
    return start + pre + chunks_per_est
