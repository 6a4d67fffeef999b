"""CPU checks of the C ABI library (no GPU compute): it loads, exports exactly
the functions include/hw_b200.h declares, its struct layouts match the
header and the Python mirrors, hw_config_default() holds the reference's
configuration defaults, hw_config_validate() rejects what the reference's
config validation rejects, and the product path fails loudly (no CPU
fallback) where there is no CUDA device.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from hw_b200 import abi, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "hw_b200.h")


def test_library_exports_every_header_function():
    L = native.lib()
    names = native.exported_symbols()
    assert len(names) >= 40
    for n in names:
        assert hasattr(L, n), n
    # and nothing else under the hw_ prefix
    out = subprocess.run(["nm", "-D", "--defined-only", native.LIB_PATH], capture_output=True, text=True,
                         check=True).stdout
    exported = sorted({ln.split()[-1] for ln in out.splitlines() if ln.split() and ln.split()[-1].startswith("hw_")})
    assert exported == names


def test_library_is_built_for_sm100a():
    # every object and the link are compiled for sm_100a only (no PTX for a
    # JIT to pick up on another architecture)
    from hw_b200 import build
    flags = build.NVCC_FLAGS
    i = flags.index("-gencode")
    assert flags[i + 1] == "arch=compute_100a,code=sm_100a"
    assert flags.count("-gencode") == 1
    assert "--use_fast_math" not in flags and "-fmad=false" in flags


_PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "hw_b200.h"
#define S(T) printf("size %s %zu\n", #T, sizeof(T));
#define O(T, m) printf("off %s.%s %zu\n", #T, #m, offsetof(T, m));
int main(void) {
  S(hw_config) S(hw_analog) S(hw_stat_accum_state) S(hw_autocorr_accum_state) S(hw_baseliner_stats)
  S(hw_lane_analog_mode) S(hw_lane_model) S(hw_lane_histogram) S(hw_lane_hist_bounds) S(hw_pulse)
  S(hw_dme_diag) S(hw_frame_interval) S(hw_gen_params) S(hw_pool_chunk) S(hw_fused_tuning)
  S(hw_basecalling_metrics) S(hw_sensor_packet) S(hw_baz_field) S(hw_prelim_hq_config) S(hw_baz_checkpoint)
  S(hw_spider_metric_block) S(hw_metric_checkpoint)
  O(hw_baseliner_stats, full_autocorr) O(hw_baseliner_stats, trace_min) O(hw_baseliner_stats, trace_max)
  O(hw_baseliner_stats, baseline_stats) O(hw_baseliner_stats, raw_baseline_sum) O(hw_baseliner_stats, background_stats)
  O(hw_lane_model, analogs) O(hw_lane_model, baseline) O(hw_lane_model, confidence)
  O(hw_lane_histogram, bin_count) O(hw_pulse, start) O(hw_pulse, width) O(hw_pulse, mean_signal)
  O(hw_pulse, mid_signal) O(hw_pulse, max_signal) O(hw_pulse, signal_m2) O(hw_pulse, label) O(hw_pulse, is_reject)
  O(hw_dme_diag, lane_iterations)
  O(hw_pool_chunk, d_trace8) O(hw_pool_chunk, d_overflows) O(hw_pool_chunk, d_metrics)
  O(hw_pool_chunk, first_frame) O(hw_pool_chunk, estimated) O(hw_pool_chunk, metrics_emitted)
  O(hw_fused_tuning, labeler_lanes_per_cta)
  O(hw_basecalling_metrics, num_pulse_frames) O(hw_basecalling_metrics, pk_mid_signal)
  O(hw_basecalling_metrics, num_pk_mid_frames) O(hw_basecalling_metrics, frame_baseline_dws)
  O(hw_basecalling_metrics, start_frame) O(hw_basecalling_metrics, autocorrelation)
  O(hw_basecalling_metrics, pixel_checksum)
  O(hw_sensor_packet, start_zmw) O(hw_sensor_packet, num_blocks)
  O(hw_baz_field, transform) O(hw_baz_field, num_bits) O(hw_baz_field, overflow_bytes)
  O(hw_prelim_hq_config, hq_throttle_fraction) O(hw_prelim_hq_config, zmw_stride)
  O(hw_baz_checkpoint, d_hq) O(hw_baz_checkpoint, num_hq) O(hw_baz_checkpoint, block)
  O(hw_prelim_hq_config, metrics) O(hw_spider_metric_block, pulse_detection_score)
  O(hw_spider_metric_block, activity_label) O(hw_spider_metric_block, pkmid) O(hw_spider_metric_block, pkzvar)
  O(hw_spider_metric_block, num_baseline_frames) O(hw_metric_checkpoint, d_offsets) O(hw_metric_checkpoint, block)
  O(hw_config, analogs) O(hw_config, filter_type) O(hw_config, max_calls_per_zmw) O(hw_config, xsp_amp_thresh)
  O(hw_config, model_estimation_mode) O(hw_config, static_baseline_variance)
  return 0;
}
"""


@pytest.fixture(scope="module")
def layout(tmp_path_factory):
    d = tmp_path_factory.mktemp("probe")
    src = d / "probe.c"
    src.write_text(_PROBE)
    exe = d / "probe"
    subprocess.run(["/usr/bin/gcc", "-std=c11", "-I", os.path.dirname(HEADER), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    sizes, offs = {}, {}
    for ln in out.splitlines():
        kind, name, val = ln.split()
        (sizes if kind == "size" else offs)[name] = int(val)
    return sizes, offs


def test_struct_sizes_match_reference_lane_types(layout):
    sizes, _ = layout
    for name, (dt, nbytes) in abi.SIZES.items():
        assert sizes[name] == nbytes == dt.itemsize, name
    assert sizes["hw_config"] == C.sizeof(abi.Config)
    assert sizes["hw_analog"] == C.sizeof(abi.Analog)
    assert sizes["hw_gen_params"] == C.sizeof(abi.GenParams)
    assert sizes["hw_frame_interval"] == C.sizeof(abi.FrameInterval)


def test_struct_offsets_match_python_mirrors(layout):
    _, offs = layout
    for key, off in offs.items():
        t, m = key.split(".")
        if t == "hw_config":
            assert getattr(abi.Config, m).offset == off, key
            continue
        dt = {"hw_baseliner_stats": abi.BLSTATS_DT, "hw_lane_model": abi.LANE_MODEL_DT,
              "hw_lane_histogram": abi.LANE_HIST_DT, "hw_pulse": abi.PULSE_DT,
              "hw_dme_diag": abi.DME_DIAG_DT, "hw_pool_chunk": abi.POOL_CHUNK_DT,
              "hw_fused_tuning": abi.FUSED_TUNING_DT, "hw_basecalling_metrics": abi.BASECALLING_METRICS_DT,
              "hw_sensor_packet": abi.SENSOR_PACKET_DT, "hw_baz_field": abi.BAZ_FIELD_DT,
              "hw_prelim_hq_config": abi.PRELIM_HQ_CONFIG_DT, "hw_baz_checkpoint": abi.BAZ_CHECKPOINT_DT,
              "hw_spider_metric_block": abi.SPIDER_METRIC_BLOCK_DT,
              "hw_metric_checkpoint": abi.METRIC_CHECKPOINT_DT}[t]
        assert dt.fields[m][1] == off, key


def _default():
    c = abi.Config()
    native.check(native.lib().hw_config_default(C.byref(c)))
    return c


def test_config_defaults_are_reference_defaults():
    """dataTypes/configs/Basecaller*Config.h PB_CONFIG_PARAM defaults."""
    c = _default()
    f32 = np.float32
    # BasecallerBaselinerConfig.h:48-89
    assert c.filter_type == abi.FILTER_TYPES["MultiScaleLarge"]
    assert (c.mean_bias_adjust, c.sigma_bias_adjust, c.mean_ema_scale_strides) == (0.0, 0.0, 0.0)
    assert c.sigma_ema_scale_strides == 512.0 and c.jump_suppression == 0.0
    # BasecallerTraceHistogramConfig.h:57-72
    assert f32(c.bin_size_coeff) == f32(0.2) and c.bin_size_low_bound_coeff == 1.0
    assert c.baseline_stat_min_frame_count == 50 and c.fallback_baseline_sigma == 10.0
    # BasecallerDmeConfig.h:90-198
    assert f32(c.analog_mix_fraction_threshold[0]) == f32(0.039) / f32(3)
    assert f32(c.analog_mix_fraction_threshold[1]) == f32(0.039)
    assert c.scale_snr_conf_tol == 1.0 and c.em_iteration_limit == 20 and c.gtest_stat_factor == -1.0
    assert c.iterate_to_limit == 0
    assert (c.min_analog_snr_thresh0, c.min_analog_snr_thresh1) == (2.0, 4.0)
    assert c.pulse_amp_regularization == 0.0 and c.model_update_method == 1
    assert c.snr_drop_thresh == 1.0 and f32(c.success_confidence_thresh) == f32(0.10)
    assert (c.confidence_half_life[0], c.confidence_half_life[1]) == (4096.0, 12000.0)
    assert c.min_frames_for_estimate == 4000 and c.num_frames_pre_accum_stats == 1000
    # BasecallerFrameLabelerConfig.h:43-60
    assert (c.viterbi_alpha, c.viterbi_beta, c.viterbi_gamma) == (1.0, 1.0, 1.0)
    assert c.roi_filter_type == 0 and (c.roi_upper_threshold, c.roi_lower_threshold) == (7.0, 2.0)
    # BasecallerPulseAccumConfig.h:89-98
    assert c.max_calls_per_zmw == 48 and c.xsp_amp_thresh == 0.70 and f32(c.xsp_width_thresh) == f32(3.5)
    # BasecallerAlgorithmConfig.h:65, StaticDetModelConfig.h:43-44
    assert c.model_estimation_mode == abi.DYNAMIC_ESTIMATIONS
    assert (c.static_baseline_mean, c.static_baseline_variance) == (0.0, 33.0)
    assert native.lib().hw_config_validate(C.byref(c)) == 0


@pytest.mark.parametrize("field, value", [
    ("filter_type", 99), ("sigma_ema_scale_strides", -1.0), ("mean_ema_scale_strides", -1.0),
    ("jump_suppression", -1.0), ("bin_size_coeff", 0.0), ("fallback_baseline_sigma", 0.0),
    ("model_update_method", 3), ("xsp_amp_thresh", 1.5), ("xsp_width_thresh", -1.0),
    ("max_calls_per_zmw", 0), ("photoelectron_sensitivity", 0.0), ("roi_filter_type", 7),
    ("model_estimation_mode", 9)])
def test_config_validation_rejects(field, value):
    c = _default()
    setattr(c, field, value)
    rc = native.lib().hw_config_validate(C.byref(c))
    assert rc == 1, (field, rc)       # HW_ERR_INVALID_ARG
    assert native.lib().hw_last_error_string()


def test_config_validation_rejects_bad_analogs():
    c = _default()
    c.analogs[2].rel_amplitude = 0.0
    assert native.lib().hw_config_validate(C.byref(c)) == 1
    c = _default()
    c.analogs[1].base_label = b"X"
    assert native.lib().hw_config_validate(C.byref(c)) == 1


def test_latent_frames():
    assert native.lib().hw_labeler_latent_frames() == abi.LATENT_FRAMES == 24


def test_version_string():
    v = native.lib().hw_version().decode()
    assert "hw_b200" in v and "sm_100a" in v


@pytest.mark.skipif("torch" in sys.modules and __import__("torch").cuda.is_available(),
                    reason="checks the no-device failure path")
def _has_device():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_device(), reason="checks the behaviour without a CUDA device")
def test_no_cpu_fallback_without_device():
    """With no CUDA device the handles cannot be created: the call returns a
    CUDA status instead of computing on the CPU."""
    from hw_b200 import workloads
    cfg = workloads.small_config()
    h = C.c_void_p()
    rc = native.lib().hw_baseliner_create(C.byref(cfg), 0, 1, 512, C.byref(h))
    assert rc != 0
    assert b"CUDA" in native.lib().hw_last_error_string() or b"cuda" in native.lib().hw_last_error_string()


@pytest.mark.skipif(_has_device(), reason="checks the behaviour without a CUDA device")
def test_fused_engine_needs_a_device_and_checks_its_arguments():
    """hw_fused_create rejects bad pool tables before touching the device and,
    with no CUDA device, returns a CUDA status (no CPU path)."""
    from hw_b200 import workloads
    cfg = workloads.small_config()
    h = C.c_void_p()
    lanes = np.array([1, 2], np.uint32)
    bad = np.array([512, 100], np.uint32)          # not a multiple of the aggregate stride
    assert native.lib().hw_fused_create(C.byref(cfg), 2, None, abi.ptr(lanes), abi.ptr(bad), C.byref(h)) == 1
    good = np.array([512, 128], np.uint32)
    rc = native.lib().hw_fused_create(C.byref(cfg), 2, None, abi.ptr(lanes), abi.ptr(good), C.byref(h))
    assert rc == 2 and b"CUDA" in native.lib().hw_last_error_string().upper()
