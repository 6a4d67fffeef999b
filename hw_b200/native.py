"""Loads libhw_b200.so and declares the C ABI of include/hw_b200.h.

The product path has no CPU fallback: if the shared library is missing or
cannot be loaded, every call raises.
"""
import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhw_b200.so")

_lib = None


class HwError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"hw_b200 CUDA library not built: {LIB_PATH} (run python -m hw_b200.build)")
    L = C.CDLL(LIB_PATH)
    vp, i32, u32 = C.c_void_p, C.c_int32, C.c_uint32
    FI = abi.FrameInterval
    PCFG = C.POINTER(abi.Config)
    PPV = C.POINTER(C.c_void_p)
    sigs = {
        "hw_last_error_string": ([], C.c_char_p),
        "hw_version": ([], C.c_char_p),
        "hw_config_default": ([PCFG], C.c_int),
        "hw_config_validate": ([PCFG], C.c_int),
        "hw_transition_matrix": ([PCFG, vp], C.c_int),
        "hw_labeler_latent_frames": ([], u32),
        "hw_baseliner_create": ([PCFG, u32, u32, u32, PPV], C.c_int),
        "hw_baseliner_destroy": ([vp], C.c_int),
        "hw_baseliner_startup_latency": ([vp, C.POINTER(u32)], C.c_int),
        "hw_baseliner_process": ([vp, vp, i32, vp, vp, vp], C.c_int),
        "hw_baseliner_process_u8": ([vp, vp, i32, vp, vp, vp], C.c_int),
        "hw_analyzer_process_u8": ([vp, vp, i32, vp, vp, vp, C.POINTER(i32), C.POINTER(i32), vp], C.c_int),
        "hw_blstats_aggregator_create": ([u32, u32, PPV], C.c_int),
        "hw_blstats_aggregator_destroy": ([vp], C.c_int),
        "hw_blstats_aggregator_add": ([vp, vp, FI, vp], C.c_int),
        "hw_blstats_aggregator_get": ([vp, vp, C.POINTER(FI), vp], C.c_int),
        "hw_blstats_aggregator_reset": ([vp, vp], C.c_int),
        "hw_histogram_create": ([PCFG, u32, u32, PPV], C.c_int),
        "hw_histogram_destroy": ([vp], C.c_int),
        "hw_histogram_add_batch": ([vp, vp, u32, FI, vp, vp], C.c_int),
        "hw_histogram_reset_from_stats": ([vp, vp, vp], C.c_int),
        "hw_histogram_reset_from_bounds": ([vp, vp, vp], C.c_int),
        "hw_histogram_get": ([vp, vp, C.POINTER(FI), vp], C.c_int),
        "hw_dme_create": ([PCFG, u32, u32, PPV], C.c_int),
        "hw_dme_destroy": ([vp], C.c_int),
        "hw_dme_init_models": ([vp, vp, vp, vp], C.c_int),
        "hw_dme_estimate": ([vp, vp, vp, FI, FI, vp, vp, vp], C.c_int),
        "hw_dme_estimate_noalloc": ([PCFG, u32, vp, vp, FI, FI, vp, vp, vp], C.c_int),
        "hw_dme_profile_phases": ([vp, C.c_int], C.c_int),
        "hw_dme_phase_cycles": ([vp, vp, vp], C.c_int),
        "hw_detection_model_import": ([vp, u32, vp, vp], C.c_int),
        "hw_detection_model_export": ([vp, u32, vp, vp], C.c_int),
        "hw_detection_model_evolve_confidence": ([vp, u32, FI, FI, C.c_float, vp], C.c_int),
        "hw_dme_estimate_proposal": ([vp, vp, vp, FI, FI, vp, vp, vp, vp], C.c_int),
        "hw_analyzer_set_learned_init": ([vp, vp], C.c_int),
        "hw_pool_set_create": ([PCFG, u32, vp, vp, PPV], C.c_int),
        "hw_pool_set_destroy": ([vp], C.c_int),
        "hw_pool_set_layout": ([vp, vp, C.POINTER(C.c_uint64), C.POINTER(u32)], C.c_int),
        "hw_pool_set_process": ([vp, vp, i32, vp, vp, vp], C.c_int),
        "hw_pool_set_outputs": ([vp, u32, PPV, PPV, PPV], C.c_int),
        "hw_fused_create": ([PCFG, u32, vp, vp, vp, PPV], C.c_int),
        "hw_fused_destroy": ([vp], C.c_int),
        "hw_chunk_fused": ([vp, vp, u32, vp], C.c_int),
        "hw_fused_set_overlap": ([vp, i32], C.c_int),
        "hw_fused_set_learned_init": ([vp, vp], C.c_int),
        "hw_fused_finish": ([vp, vp], C.c_int),
        "hw_fused_use_graphs": ([vp, i32], C.c_int),
        "hw_fused_set_tuning": ([vp, vp, u32], C.c_int),
        "hw_fused_models": ([vp, u32, vp, C.POINTER(FI), vp], C.c_int),
        "hw_fused_last_diag": ([vp, u32, vp, C.POINTER(i32), vp], C.c_int),
        "hw_fused_last_step": ([vp, C.POINTER(u32), C.POINTER(u32)], C.c_int),
        "hw_fused_profile": ([vp, i32], C.c_int),
        "hw_repacker_create": ([u32, u32, u32, i32, PPV], C.c_int),
        "hw_repacker_destroy": ([vp], C.c_int),
        "hw_repacker_num_pools": ([vp, C.POINTER(u32)], C.c_int),
        "hw_repack_chunk": ([vp, vp, u32, vp, i32, vp, vp], C.c_int),
        "hw_baz_preset": ([i32, vp, C.POINTER(u32), C.POINTER(i32)], C.c_int),
        "hw_baz_encoder_create": ([vp, u32, i32, u32, PPV], C.c_int),
        "hw_baz_encoder_destroy": ([vp], C.c_int),
        "hw_baz_encoder_set_zmw_stride": ([vp, u32], C.c_int),
        "hw_baz_encoder_set_wait_limit": ([vp, u32, i32], C.c_int),
        "hw_pulse_compactor_create": ([u32, PPV], C.c_int),
        "hw_pulse_compactor_destroy": ([vp], C.c_int),
        "hw_pulses_compact": ([vp, vp, vp, u32, vp, vp, C.POINTER(u32), vp], C.c_int),
        "hw_pulse_compactor_total": ([vp, u32, C.POINTER(C.c_uint64)], C.c_int),
        "hw_prelim_hq_config_default": ([vp], C.c_int),
        "hw_prelim_hq_create": ([vp, u32, i32, u32, vp, PPV], C.c_int),
        "hw_prelim_hq_destroy": ([vp], C.c_int),
        "hw_prelim_hq_process": ([vp, vp, vp, u32, vp, vp, C.POINTER(i32), vp, vp], C.c_int),
        "hw_prelim_hq_flush": ([vp, C.POINTER(i32), vp, vp], C.c_int),
        "hw_prelim_hq_activity": ([vp, vp, vp], C.c_int),
        "hw_prelim_hq_metrics": ([vp, vp], C.c_int),
        "hw_baz_encode": ([vp, vp, vp, u32, vp, C.c_uint64, vp, vp, C.POINTER(C.c_uint64), vp], C.c_int),
        "hw_baz_encode_async": ([vp, vp, vp, u32, vp, C.c_uint64, vp, vp, vp], C.c_int),
        "hw_baz_encode_result": ([vp, C.POINTER(C.c_uint64)], C.c_int),
        "hw_fused_enable_hf_metrics": ([vp, u32, C.c_double, i32, vp, vp, vp, vp, vp, u32, vp, C.c_float], C.c_int),
        "hw_analyzer_chunk_metrics": ([vp, vp, vp, vp, vp], C.c_int),
        "hw_hfmetrics_create": ([u32, u32, C.c_double, i32, PPV], C.c_int),
        "hw_hfmetrics_destroy": ([vp], C.c_int),
        "hw_hfmetrics_set_cart": ([vp, vp, vp, vp, vp, vp, u32, vp, C.c_float], C.c_int),
        "hw_hfmetrics_process": ([vp, vp, vp, u32, vp, vp, vp, vp, i32, u32, vp, C.POINTER(i32), vp], C.c_int),
        "hw_fused_stage_times": ([vp, vp, vp], C.c_int),
        "hw_analyzer_state_size": ([vp, C.POINTER(C.c_uint64)], C.c_int),
        "hw_analyzer_state_export": ([vp, vp, C.c_uint64, vp], C.c_int),
        "hw_analyzer_state_import": ([vp, vp, C.c_uint64, vp], C.c_int),
        "hw_dme_em_fit_scratch_bytes": ([u32, C.POINTER(C.c_uint64)], C.c_int),
        "hw_dme_em_fit": ([PCFG, u32, vp, vp, FI, FI, vp, C.c_int, vp, vp, C.c_float, u32, vp, vp, vp, vp, vp, vp],
                          C.c_int),
        "hw_learned_init_create": ([u32, C.c_uint64, PPV], C.c_int),
        "hw_learned_init_destroy": ([vp], C.c_int),
        "hw_learned_init_param_count": ([C.POINTER(u32)], C.c_int),
        "hw_learned_init_get_params": ([vp, vp, vp], C.c_int),
        "hw_learned_init_set_params": ([vp, vp, vp], C.c_int),
        "hw_learned_init_features": ([u32, vp, vp, vp, vp], C.c_int),
        "hw_learned_init_targets": ([PCFG, u32, vp, vp, vp, vp], C.c_int),
        "hw_learned_init_forward": ([vp, vp, u32, vp, vp], C.c_int),
        "hw_learned_init_forward_status": ([vp], C.c_int),
        "hw_learned_init_propose": ([vp, u32, vp, vp, vp, vp], C.c_int),
        "hw_learned_init_proposal": ([vp, u32, vp, vp, vp, vp], C.c_int),
        "hw_learned_init_gradients": ([vp, vp, vp, vp, u32, vp, C.POINTER(C.c_float), vp], C.c_int),
        "hw_learned_init_train_step": ([vp, vp, vp, vp, u32, C.c_float, C.c_float, C.POINTER(C.c_float), vp],
                                       C.c_int),
        "hw_labeler_create": ([PCFG, u32, u32, u32, PPV], C.c_int),
        "hw_labeler_destroy": ([vp], C.c_int),
        "hw_labeler_process": ([vp, vp, vp, vp, vp, vp, vp, vp], C.c_int),
        "hw_pulse_accumulator_create": ([PCFG, u32, u32, u32, PPV], C.c_int),
        "hw_pulse_accumulator_destroy": ([vp], C.c_int),
        "hw_pulse_accumulator_process": ([vp, vp, vp, vp, i32, vp, vp, vp, vp, vp, vp], C.c_int),
        "hw_analyzer_create": ([PCFG, u32, u32, u32, PPV], C.c_int),
        "hw_analyzer_destroy": ([vp], C.c_int),
        "hw_analyzer_process": ([vp, vp, i32, vp, vp, vp, C.POINTER(i32), C.POINTER(i32), vp], C.c_int),
        "hw_analyzer_models": ([vp, vp, C.POINTER(FI), vp], C.c_int),
        "hw_analyzer_last_diag": ([vp, vp, C.POINTER(i32), vp], C.c_int),
        "hw_analyzer_profile": ([vp, i32], C.c_int),
        "hw_analyzer_stage_times": ([vp, vp, vp], C.c_int),
        "hw_gen_params_default": ([C.c_int, C.POINTER(abi.GenParams)], C.c_int),
        "hw_trace_generator_create": ([C.POINTER(abi.GenParams), u32, C.c_uint64, PPV], C.c_int),
        "hw_trace_generator_destroy": ([vp], C.c_int),
        "hw_trace_generator_next": ([vp, vp, i32, u32, vp], C.c_int),
    }
    for name, (args, res) in sigs.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = res
    _lib = L
    return L


def check(rc):
    if rc != 0:
        raise HwError(rc, lib().hw_last_error_string().decode())
    return rc


def exported_symbols():
    """Names of the C ABI functions declared in include/hw_b200.h."""
    import re
    hdr = os.path.join(_HERE, os.pardir, "include", "hw_b200.h")
    text = open(hdr).read()
    return sorted(set(re.findall(r"^(?:int|const char\*|uint32_t)\s+(hw_[a-z0-9_]+)\(", text, re.M)))
