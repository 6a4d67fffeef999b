"""ctypes binding of the CPU oracle (oracle/hw_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the hw_b200 package.  The oracle is a
literal CPU restatement of the reference's Host* trace-analysis path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

from hw_b200 import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libhw_oracle.so")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, u32 = C.c_void_p, C.c_int32, C.c_uint32
        FI = abi.FrameInterval
        L.or_last_error.restype = C.c_char_p
        L.or_config_default.argtypes = [C.POINTER(abi.Config)]
        L.or_transition_matrix.argtypes = [C.POINTER(abi.Config), vp]
        L.or_pool_create.argtypes = [C.POINTER(abi.Config), u32, u32, u32]
        L.or_pool_create.restype = vp
        L.or_pool_destroy.argtypes = [vp]
        L.or_set_threads.argtypes = [C.c_int]
        L.or_baseliner_startup_latency.argtypes = [vp]
        L.or_baseliner_startup_latency.restype = u32
        L.or_baseline.argtypes = [vp, vp, i32, vp, vp]
        L.or_agg_add.argtypes = [vp, vp, FI]
        L.or_agg_get.argtypes = [vp, vp, C.POINTER(FI)]
        L.or_agg_reset.argtypes = [vp]
        L.or_hist_reset_from_stats.argtypes = [vp, vp]
        L.or_hist_reset_from_bounds.argtypes = [vp, vp]
        L.or_hist_add.argtypes = [vp, vp, u32, FI, vp]
        L.or_hist_get.argtypes = [vp, vp, C.POINTER(FI)]
        L.or_dme_init_models.argtypes = [vp, vp, vp]
        L.or_dme_estimate.argtypes = [vp, vp, vp, FI, FI, vp, vp]
        L.or_label.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.or_pulses.argtypes = [vp, vp, vp, vp, i32, vp, vp, vp, vp, vp]
        L.or_dme_estimate_proposal.argtypes = [vp, vp, vp, FI, FI, vp, vp, vp]
        L.or_em_fit.argtypes = [vp, vp, vp, FI, FI, vp, C.c_int, vp, vp, C.c_float, u32, vp, vp, vp, vp]
        L.or_static_model.argtypes = [C.POINTER(abi.Config), vp]
        L.or_extremum_stage.argtypes = [C.c_int, C.c_int, vp, C.c_int, C.c_int, vp]
        L.or_expf.argtypes = [C.c_float]
        L.or_expf.restype = C.c_float
        L.or_logf.argtypes = [C.c_float]
        L.or_logf.restype = C.c_float
        L.or_f32_to_f16.argtypes = [C.c_float]
        L.or_f32_to_f16.restype = C.c_uint16
        L.or_detection_model_import.argtypes = [vp, u32, vp]
        L.or_detection_model_export.argtypes = [vp, u32, vp]
        L.or_detection_model_evolve_confidence.argtypes = [vp, u32, FI, FI, C.c_float]
        L.or_picket_fence.argtypes = [u32, C.c_uint64, C.c_int, C.c_uint16, C.c_uint16, C.c_float, C.c_float,
                                      C.c_int16, C.c_int16, vp, C.c_int, C.c_int16, vp]
        L.or_gen_params_default.argtypes = [C.c_int, C.POINTER(abi.GenParams)]
        L.or_gen_create.argtypes = [C.POINTER(abi.GenParams), u32, C.c_uint64]
        L.or_gen_create.restype = vp
        L.or_gen_destroy.argtypes = [vp]
        L.or_gen_next.argtypes = [vp, vp, C.c_int64, u32]
        L.or_to_i16.argtypes = [C.c_float]
        L.or_to_i16.restype = C.c_int16
        L.or_hf_create.argtypes = [u32, u32, C.c_double, i32]
        L.or_hf_create.restype = vp
        L.or_hf_destroy.argtypes = [vp]
        L.or_hf_set_cart.argtypes = [vp, vp, vp, vp, vp, vp, u32, vp, C.c_float]
        L.or_hf_process.argtypes = [vp, vp, vp, u32, vp, vp, vp, vp, i32, u32, vp, C.POINTER(i32)]
        L.or_repack.argtypes = [u32, u32, u32, i32, vp, u32, vp, i32, vp]
        L.or_baz_encode_values.argtypes = [vp, u32, vp, u32, vp, C.c_uint64, vp]
        L.or_baz_encode_values.restype = C.c_int64
        L.or_baz_decode_values.argtypes = [vp, u32, vp, u32, vp, vp, C.POINTER(C.c_uint64)]
        L.or_baz_serializer_roundtrip.argtypes = [i32, i32, i32, i32, C.c_uint64, i32, C.POINTER(C.c_uint64)]
        L.or_baz_serializer_roundtrip.restype = C.c_uint64
        L.or_baz_float_fixed_roundtrip.argtypes = [C.c_float, i32, i32, i32, C.POINTER(C.c_uint64)]
        L.or_baz_float_fixed_roundtrip.restype = C.c_float
        L.or_prehq_create.argtypes = [u32, u32, i32, C.c_float]
        L.or_prehq_create.restype = vp
        L.or_prehq_destroy.argtypes = [vp]
        L.or_prehq_add.argtypes = [vp, vp, vp, vp]
        L.or_prehq_end_block.argtypes = [vp, vp, vp, C.c_uint64, vp, vp, vp]
        L.or_prehq_end_block.restype = C.c_int64
        L.or_prehq_flush.argtypes = [vp, vp, C.c_uint64, vp, vp, vp]
        L.or_prehq_flush.restype = C.c_int64
        u64 = C.c_uint64
        L.or_metrics_create.argtypes = [u32, u32, i32, u32, i32]
        L.or_metrics_create.restype = vp
        L.or_metrics_destroy.argtypes = [vp]
        L.or_metrics_add.argtypes = [vp, vp]
        L.or_metrics_end_block.argtypes = [vp, vp, vp, u64, vp]
        L.or_metrics_end_block.restype = C.c_int64
        L.or_metrics_take.argtypes = [vp, vp, u64, vp]
        L.or_metrics_take.restype = C.c_int64
        L.or_metrics_flush.argtypes = [vp, vp, u64, vp]
        L.or_metrics_flush.restype = C.c_int64
        L.or_metrics_activity.argtypes = [vp, vp]
        L.or_half_bits.argtypes = [vp, u64, vp]
        L.or_half_float.argtypes = [vp, u64, vp]
        L.or_metric_block_convert.argtypes = [vp, i32, i32, vp]
        L.or_metrics_kat.argtypes = [vp, i32, i32, i32, i32, vp, vp]
        L.or_baz_encode_chunk.argtypes = [vp, u32, i32, u32, u32, vp, vp, u32, vp, C.c_uint64, vp, vp]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"oracle: {abi.STATUS_NAMES.get(rc, rc)}: {lib().or_last_error().decode()}")


def default_config():
    c = abi.Config()
    lib().or_config_default(C.byref(c))
    return c


def transition_matrix(cfg):
    out = np.zeros((abi.NUM_STATES, abi.NUM_STATES), np.float32)
    lib().or_transition_matrix(C.byref(cfg), abi.ptr(out))
    return out


def detection_model_import(models):
    """DetectionModelHost(ldm): fp16 lane models -> float [lanes][16][64]."""
    models = np.ascontiguousarray(models)
    out = np.zeros((len(models), 16, abi.LANE), np.float32)
    _check(lib().or_detection_model_import(abi.ptr(models), len(models), abi.ptr(out)))
    return out


def detection_model_export(params):
    """ExportTo: float [lanes][16][64] -> fp16 lane models."""
    params = np.ascontiguousarray(params, np.float32)
    out = np.zeros(len(params), abi.LANE_MODEL_DT)
    _check(lib().or_detection_model_export(abi.ptr(params), len(params), abi.ptr(out)))
    return out


def detection_model_evolve_confidence(params, fi_from, fi_to, half_life):
    params = np.ascontiguousarray(params, np.float32).copy()
    _check(lib().or_detection_model_evolve_confidence(abi.ptr(params), len(params), abi.FrameInterval(*fi_from),
                                                      abi.FrameInterval(*fi_to), half_life))
    return params


def picket_fence(num_frames, idx, poisson=True, pulse_width=5, pulse_ipd=10, width_rate=0.2, ipd_rate=0.1,
                 baseline_level=200, baseline_sigma=20, levels=(200,), pedestal=0):
    """The reference's PicketFenceGenerator signal `idx` (int16, num_frames);
    defaults are its Config defaults."""
    lv = np.ascontiguousarray(levels, np.int16)
    out = np.zeros(num_frames, np.int16)
    _check(lib().or_picket_fence(num_frames, idx, int(poisson), pulse_width, pulse_ipd, width_rate, ipd_rate,
                                 baseline_level, baseline_sigma, abi.ptr(lv), len(lv), pedestal, abi.ptr(out)))
    return out


def gen_params_default(workload):
    p = abi.GenParams()
    _check(lib().or_gen_params_default(int(workload), C.byref(p)))
    return p


class TraceGenerator:
    """The workloads' trace generator on the host (byte-identical to
    hw_trace_generator): chunks [lanes][frames][64] int16, in order."""

    def __init__(self, lanes, workload=1, zmw_offset=0, params=None):
        self.lanes = lanes
        self.params = gen_params_default(workload) if params is None else params
        self.h = lib().or_gen_create(C.byref(self.params), lanes, zmw_offset)
        if not self.h:
            raise RuntimeError("oracle generator create failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_gen_destroy(self.h)
            self.h = None

    def next(self, first_frame, frames):
        out = np.empty((self.lanes, frames, abi.LANE), np.int16)
        _check(lib().or_gen_next(self.h, abi.ptr(out), int(first_frame), int(frames)))
        return out


def set_threads(n):
    return lib().or_set_threads(int(n))


class Pool:
    """All Host* filters of one pool (baseliner, aggregator, histogram, DME,
    labeler, pulse accumulator) with the reference's per-stage calls."""

    def __init__(self, cfg, lanes, frames_per_chunk, pool_id=0):
        self.cfg = cfg.copy()
        self.lanes = lanes
        self.F = frames_per_chunk
        self.h = lib().or_pool_create(C.byref(self.cfg), pool_id, lanes, frames_per_chunk)
        if not self.h:
            raise RuntimeError("oracle pool create failed: " + lib().or_last_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_pool_destroy(self.h)
            self.h = None

    def startup_latency(self):
        return lib().or_baseliner_startup_latency(self.h)

    def baseline(self, trace, first_frame):
        trace = np.ascontiguousarray(trace, dtype=np.int16)
        if trace.shape != (self.lanes, self.F, abi.LANE):
            raise ValueError(f"oracle baseline: trace {trace.shape} for {self.lanes} lanes of {self.F} frames")
        out = np.empty_like(trace)
        stats = np.zeros(self.lanes, abi.BLSTATS_DT)
        _check(lib().or_baseline(self.h, abi.ptr(trace), first_frame, abi.ptr(out), abi.ptr(stats)))
        return out, stats

    def agg_add(self, stats, fi):
        _check(lib().or_agg_add(self.h, abi.ptr(stats), abi.FrameInterval(*fi)))

    def agg_get(self):
        out = np.zeros(self.lanes, abi.BLSTATS_DT)
        fi = abi.FrameInterval()
        _check(lib().or_agg_get(self.h, abi.ptr(out), C.byref(fi)))
        return out, fi.tuple()

    def agg_reset(self):
        _check(lib().or_agg_reset(self.h))

    def hist_reset_from_stats(self, stats):
        _check(lib().or_hist_reset_from_stats(self.h, abi.ptr(stats)))

    def hist_reset_from_bounds(self, bounds):
        _check(lib().or_hist_reset_from_bounds(self.h, abi.ptr(bounds)))

    def hist_add(self, traces, fi, models):
        traces = np.ascontiguousarray(traces, dtype=np.int16)
        frames = traces.shape[1]
        _check(lib().or_hist_add(self.h, abi.ptr(traces), frames, abi.FrameInterval(*fi), abi.ptr(models)))

    def hist_get(self):
        out = np.zeros(self.lanes, abi.LANE_HIST_DT)
        fi = abi.FrameInterval()
        _check(lib().or_hist_get(self.h, abi.ptr(out), C.byref(fi)))
        return out, fi.tuple()

    def init_models(self, stats):
        out = np.zeros(self.lanes, abi.LANE_MODEL_DT)
        _check(lib().or_dme_init_models(self.h, abi.ptr(stats), abi.ptr(out)))
        return out

    def estimate(self, hist, stats, hist_fi, model_fi, models):
        models = models.copy()
        diag = np.zeros(self.lanes, abi.DME_DIAG_DT)
        _check(lib().or_dme_estimate(self.h, abi.ptr(hist), abi.ptr(stats), abi.FrameInterval(*hist_fi),
                                     abi.FrameInterval(*model_fi), abi.ptr(models), abi.ptr(diag)))
        return models, diag

    def estimate_proposal(self, hist, stats, hist_fi, model_fi, models, proposal):
        """Estimate from a learned start (see hw_dme_estimate_proposal)."""
        models = models.copy()
        diag = np.zeros(self.lanes, abi.DME_DIAG_DT)
        prop = np.ascontiguousarray(proposal, np.float32)
        _check(lib().or_dme_estimate_proposal(self.h, abi.ptr(hist), abi.ptr(stats), abi.FrameInterval(*hist_fi),
                                              abi.FrameInterval(*model_fi), abi.ptr(models), abi.ptr(diag),
                                              abi.ptr(prop)))
        return models, diag

    def em_fit(self, hist, stats, hist_fi, model_fi, models, mode=0, proposal=None, target=None, tol=1e-4,
               max_iter=20, at_stop=False):
        """Single-ZMW EM fit (see hw_dme_em_fit): returns params [lanes][15][64],
        iters [lanes][5][64] and log-likelihoods [lanes][3][64], and with
        at_stop=True the parameters at the first converged iteration."""
        stop = np.zeros((self.lanes, 15, abi.LANE), np.float32) if at_stop else None
        params = np.zeros((self.lanes, 15, abi.LANE), np.float32)
        iters = np.zeros((self.lanes, 5, abi.LANE), np.int32)
        ll = np.zeros((self.lanes, 3, abi.LANE), np.float32)
        prop = None if proposal is None else np.ascontiguousarray(proposal, np.float32)
        tgt = None if target is None else np.ascontiguousarray(target, np.float32)
        _check(lib().or_em_fit(self.h, abi.ptr(hist), abi.ptr(stats), abi.FrameInterval(*hist_fi),
                               abi.FrameInterval(*model_fi), abi.ptr(models), int(mode), abi.ptr(prop), abi.ptr(tgt),
                               float(tol), int(max_iter), abi.ptr(params), abi.ptr(iters), abi.ptr(ll),
                               abi.ptr(stop)))
        return (params, iters, ll, stop) if at_stop else (params, iters, ll)

    def label(self, traces, models, margin=False):
        """FrameLabeler: labels, latent trace, Viterbi score (and, with
        margin=True, the best path's decision margin of every label)."""
        traces = np.ascontiguousarray(traces, dtype=np.int16)
        if traces.shape != (self.lanes, self.F, abi.LANE) or len(models) != self.lanes:
            raise ValueError(f"oracle label: traces {traces.shape}, {len(models)} models for "
                             f"{self.lanes} lanes of {self.F} frames")
        labels = np.empty_like(traces)
        lat = np.empty((self.lanes, abi.LATENT_FRAMES, abi.LANE), np.int16)
        score = np.empty((self.lanes, abi.LANE), np.float32)
        mg = np.empty(traces.shape, np.float32) if margin else None
        _check(lib().or_label(self.h, abi.ptr(traces), abi.ptr(models), abi.ptr(labels), abi.ptr(lat),
                              abi.ptr(score), abi.ptr(mg) if margin else None))
        return (labels, lat, score, mg) if margin else (labels, lat, score)

    def pulses(self, labels, latent, traces, first_frame, models):
        cap = self.cfg.max_calls_per_zmw
        pulses = np.zeros((self.lanes, abi.LANE, cap), abi.PULSE_DT)
        lens = np.zeros((self.lanes, abi.LANE), np.uint32)
        ovf = np.zeros((self.lanes, abi.LANE), np.uint32)
        bls = np.zeros(self.lanes, abi.STAT_ACCUM_DT)
        labels, latent, traces = (np.ascontiguousarray(labels), np.ascontiguousarray(latent),
                                  np.ascontiguousarray(traces))      # held until the call returns
        _check(lib().or_pulses(self.h, abi.ptr(labels), abi.ptr(latent),
                               abi.ptr(traces), first_frame, abi.ptr(models),
                               abi.ptr(pulses), abi.ptr(lens), abi.ptr(ovf), abi.ptr(bls)))
        return pulses, lens, ovf, bls


def expf(x):
    return lib().or_expf(float(x))


def logf(x):
    return lib().or_logf(float(x))


def extremum_stage(width, is_max, blocks):
    """One window stage (stride 1) over blocks[chunks][F][64] of one lane."""
    blocks = np.ascontiguousarray(blocks, dtype=np.int16)
    out = np.empty_like(blocks)
    _check(lib().or_extremum_stage(int(width), int(bool(is_max)), abi.ptr(blocks), blocks.shape[1],
                                   blocks.shape[0], abi.ptr(out)))
    return out


def static_model(cfg, lanes):
    """The FixedModelBatchAnalyzer detection model for `lanes` lanes."""
    one = np.zeros(1, abi.LANE_MODEL_DT)
    _check(lib().or_static_model(C.byref(cfg), abi.ptr(one)))
    return np.repeat(one, lanes)


class HfMetrics:
    """HFMetricsFilterHost of one pool (oracle)."""

    def __init__(self, lanes, frames_per_block=4096, frame_rate=100.0, realtime_activity_labels=True):
        self.lanes = lanes
        self.h = lib().or_hf_create(lanes, frames_per_block, frame_rate, int(bool(realtime_activity_labels)))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_hf_destroy(self.h)
            self.h = None

    def set_cart(self, cart):
        """cart: mapping with children_left/right, feature, threshold, value,
        hsw_curve, max_acceptable_halfsandwich_rate (hw_b200/data/trained_cart.npz)."""
        self._cart = {k: np.ascontiguousarray(cart[k]) for k in cart}
        c = self._cart
        _check(lib().or_hf_set_cart(self.h, abi.ptr(c["children_left"]), abi.ptr(c["children_right"]),
                                    abi.ptr(c["feature"]), abi.ptr(c["threshold"]), abi.ptr(c["value"]),
                                    len(c["children_left"]), abi.ptr(c["hsw_curve"]),
                                    float(np.asarray(c["max_acceptable_halfsandwich_rate"]).reshape(-1)[0])))

    def process(self, pulses, lens, baseliner_stats, models, viterbi, pd_stats, first_frame, frames):
        """Returns the block's metrics (numpy BASECALLING_METRICS_DT [lanes]) or None."""
        # converted copies held in locals until the call returns
        pulses = np.ascontiguousarray(pulses)
        lens = np.ascontiguousarray(lens, np.uint32)
        baseliner_stats = np.ascontiguousarray(baseliner_stats)
        models = np.ascontiguousarray(models)
        viterbi = np.ascontiguousarray(viterbi, np.float32)
        pd_stats = np.ascontiguousarray(pd_stats)
        cap = pulses.shape[-1]
        out = np.zeros(self.lanes, abi.BASECALLING_METRICS_DT)
        em = C.c_int32()
        _check(lib().or_hf_process(self.h, abi.ptr(pulses), abi.ptr(lens), cap, abi.ptr(baseliner_stats),
                                   abi.ptr(models), abi.ptr(viterbi), abi.ptr(pd_stats), int(first_frame),
                                   int(frames), abi.ptr(out), C.byref(em)))
        return out if em.value else None


def repack(num_zmw, lanes_per_pool, frames_per_chunk, encoding, packets, data, chunk_first_frame, pool_chunks):
    """BatchFiller::Process over a chunk's packets (abi.SENSOR_PACKET_DT table,
    uint8 packet data); pool_chunks: list of numpy arrays updated in place."""
    packets = np.ascontiguousarray(packets, abi.SENSOR_PACKET_DT)
    data = np.ascontiguousarray(data, np.uint8)
    ptrs = (C.c_void_p * len(pool_chunks))(*[c.ctypes.data for c in pool_chunks])
    _check(lib().or_repack(num_zmw, lanes_per_pool, frames_per_chunk, encoding, abi.ptr(packets), len(packets),
                           abi.ptr(data), int(chunk_first_frame), ptrs))


# the field values of one pulse (struct BazPulse of the oracle)
BAZ_PULSE_DT = np.dtype([("label", np.uint8), ("start", np.uint32), ("width", np.uint16), ("is_base", np.uint8),
                         ("pkmax", np.float32), ("pkmid", np.float32), ("pkmean", np.float32),
                         ("pkvar", np.float32)], align=True)


def baz_encode_values(fields, pulses, last=None):
    """One ZMW's pulses (BAZ_PULSE_DT) encoded with the field list; `last`
    (uint64 per field, delta state) is updated.  Returns the bytes."""
    fields = np.ascontiguousarray(fields, abi.BAZ_FIELD_DT)
    pulses = np.ascontiguousarray(pulses, BAZ_PULSE_DT)
    last = np.zeros(len(fields), np.uint64) if last is None else last
    cap = 64 * len(pulses) * len(fields) + 64
    out = np.zeros(cap, np.uint8)
    n = lib().or_baz_encode_values(abi.ptr(fields), len(fields), abi.ptr(pulses), len(pulses), abi.ptr(out), cap,
                                   abi.ptr(last))
    if n < 0:
        raise RuntimeError("oracle: BAZ buffer too small")
    return out[:n].copy()


def baz_serializer_roundtrip(serialize, num_bits, overflow_bytes, signed, value, mask=True):
    """One serializer: (decoded value as uint64, overflow bytes of the value)."""
    ov = C.c_uint64()
    r = lib().or_baz_serializer_roundtrip(serialize, num_bits, overflow_bytes, int(signed), value & (2**64 - 1),
                                          int(mask), C.byref(ov))
    return r, ov.value


def baz_float_fixed_roundtrip(v, signed, scale, nbytes):
    """FloatFixedCodec: (reverted float, code)."""
    code = C.c_uint64()
    r = lib().or_baz_float_fixed_roundtrip(float(v), int(signed), scale, nbytes, C.byref(code))
    return np.float32(r), code.value


def baz_decode_values(fields, data, n, last=None):
    """Inverse of baz_encode_values: (pulses, bytes consumed)."""
    fields = np.ascontiguousarray(fields, abi.BAZ_FIELD_DT)
    data = np.ascontiguousarray(data, np.uint8)
    last = np.zeros(len(fields), np.uint64) if last is None else last
    out = np.zeros(n, BAZ_PULSE_DT)
    used = C.c_uint64()
    _check(lib().or_baz_decode_values(abi.ptr(fields), len(fields), abi.ptr(data), n, abi.ptr(out), abi.ptr(last),
                                      C.byref(used)))
    return out, used.value


class BazEncoder:
    """PrelimHQFilter + PacketBuffer::AddZmw over chunks of the basecaller's
    pulses ([num_zmw][cap] abi.PULSE_DT); per-ZMW delta state kept."""

    def __init__(self, fields, skip_rejects, num_zmw, zmw_stride=1):
        self.fields = np.ascontiguousarray(fields, abi.BAZ_FIELD_DT)
        self.skip = int(bool(skip_rejects))
        self.num_zmw = num_zmw
        self.stride = zmw_stride
        self.last = np.zeros((num_zmw, len(self.fields)), np.uint64)

    def __call__(self, pulses, lens, cap):
        pulses = np.ascontiguousarray(pulses, abi.PULSE_DT)
        lens = np.ascontiguousarray(lens, np.uint32)
        out_cap = int(lens.sum()) * (8 * len(self.fields) + 8) + 16
        out = np.zeros(out_cap, np.uint8)
        offsets = np.zeros(self.num_zmw + 1, np.uint64)
        _check(lib().or_baz_encode_chunk(abi.ptr(self.fields), len(self.fields), self.skip, self.num_zmw,
                                         self.stride, abi.ptr(pulses), abi.ptr(lens), int(cap), abi.ptr(out), out_cap,
                                         abi.ptr(offsets), abi.ptr(self.last)))
        return out[:int(offsets[-1])].copy(), offsets


class PrelimHq:
    """PacketBufferManager checkpoints + DummyPreHQ marking (the preliminary HQ
    stage) over per-chunk encoded bytes: add() a chunk's (bytes, offsets,
    events), end_block() at each metric block's end."""

    def __init__(self, num_zmw, lookback, enable, throttle=0.1):
        self.n = num_zmw
        self.h = lib().or_prehq_create(num_zmw, lookback, int(bool(enable)), float(throttle))

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_prehq_destroy(self.h)
            self.h = None

    def add(self, data, offsets, events):
        data = np.ascontiguousarray(data, np.uint8)
        offsets = np.ascontiguousarray(offsets, np.uint64)
        events = np.ascontiguousarray(events, np.uint32)
        lib().or_prehq_add(self.h, abi.ptr(data) if len(data) else None, abi.ptr(offsets), abi.ptr(events))

    def _out(self, fn, *args):
        cap = 1 << 16
        while True:
            out = np.zeros(cap, np.uint8)
            off = np.zeros(self.n + 1, np.uint64)
            ev = np.zeros(self.n, np.uint32)
            hq = np.zeros(self.n, np.uint8)
            n = fn(self.h, *args, abi.ptr(out), cap, abi.ptr(off), abi.ptr(ev), abi.ptr(hq))
            if n >= 0:
                return out[:n].copy(), off, ev, hq
            cap *= 4

    def end_block(self, marks=None):
        """(bytes, offsets[n + 1], events[n], hq[n]) of the block's checkpoint."""
        m = None if marks is None else np.ascontiguousarray(marks, np.uint8)
        return self._out(lib().or_prehq_end_block, abi.ptr(m) if m is not None else None)

    def flush(self):
        return self._out(lib().or_prehq_flush)


def half_bits(x):
    """float32 -> IEEE half bits as the reference's half type rounds them."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty(x.shape, np.uint16)
    lib().or_half_bits(abi.ptr(x), x.size, abi.ptr(out))
    return out


def half_float(bits):
    bits = np.ascontiguousarray(bits, np.uint16)
    out = np.empty(bits.shape, np.float32)
    lib().or_half_float(abi.ptr(bits), bits.size, abi.ptr(out))
    return out


METRIC_KINDS = {"production_half": 0, "complete_half": 1, "production_float": 2, "complete_float": 3}


def metric_block(lane, z, kind):
    """One ZMW of a lane's BasecallingMetrics (abi.BASECALLING_METRICS_DT)
    through one of the reference's metric types, converted."""
    lane = np.ascontiguousarray(lane, abi.BASECALLING_METRICS_DT)
    out = np.zeros(1, abi.SPIDER_METRIC_BLOCK_DT)
    lib().or_metric_block_convert(abi.ptr(lane), int(z), METRIC_KINDS[kind], abi.ptr(out))
    return out[0]


def metrics_kat(lane, test, z0=0, z1=1, reps=1):
    """The aggregation sequences of the reference's metric known-answer
    tests (or_metrics_kat): (converted block, raw aggregate fields)."""
    lane = np.ascontiguousarray(lane, abi.BASECALLING_METRICS_DT)
    out = np.zeros(1, abi.SPIDER_METRIC_BLOCK_DT)
    raw = np.zeros(20, np.float64)
    lib().or_metrics_kat(abi.ptr(lane), int(test), int(z0), int(z1), int(reps), abi.ptr(out), abi.ptr(raw))
    return out[0], raw


class MetricSide:
    """MetricBufferManager of the preliminary HQ stage: add() one block's HF
    metrics (lanes of abi.BASECALLING_METRICS_DT), end_block(newly) at each
    metric block's end, flush() at the end.  `literal` keeps the reference's
    two index slips (see hw_oracle.cpp)."""

    def __init__(self, num_zmw, lookback, enable_prehq, zmw_stride=1, literal=False):
        self.n = num_zmw
        self.h = lib().or_metrics_create(num_zmw, lookback, int(bool(enable_prehq)), zmw_stride, int(bool(literal)))
        if not self.h:
            raise ValueError("or_metrics_create: bad argument")

    def __del__(self):
        if getattr(self, "h", None):
            lib().or_metrics_destroy(self.h)
            self.h = None

    def add(self, lanes):
        lanes = np.ascontiguousarray(lanes, abi.BASECALLING_METRICS_DT)
        assert len(lanes) * abi.LANE >= self.n
        lib().or_metrics_add(self.h, abi.ptr(lanes))

    def _take(self, fn, *args):
        cap = max(1024, self.n * 2)
        off = np.zeros(self.n + 1, np.uint64)
        while True:
            out = np.zeros(cap, abi.SPIDER_METRIC_BLOCK_DT)
            k = fn(self.h, *args, abi.ptr(out), cap, abi.ptr(off))
            if k >= 0:
                return out[:k].copy(), off
            fn, args = lib().or_metrics_take, ()
            cap *= 4

    def end_block(self, newly=None):
        """(blocks, offsets[n + 1]) of the block's metric checkpoint."""
        m = None if newly is None else np.ascontiguousarray(newly, np.uint8)
        return self._take(lib().or_metrics_end_block, abi.ptr(m) if m is not None else None)

    def flush(self):
        return self._take(lib().or_metrics_flush)

    def activity(self):
        out = np.zeros(self.n, np.uint8)
        lib().or_metrics_activity(self.h, abi.ptr(out))
        return out
