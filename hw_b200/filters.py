"""Host-side mirrors of the reference's per-pool filter interfaces.

Each class wraps one C-ABI handle and keeps the reference's method names and
argument meaning (src/basecaller/basecaller/traceAnalysis):

  Baseliner                  Baseliner.h:53-79 (operator(), StartupLatency)
  BaselineStatsAggregator    BaselineStatsAggregator.h:45-104
  TraceHistogramAccumulator  TraceHistogramAccumulator.h:96-154
  DmeEmEstimator             CoreDMEstimator.h:151-162 (InitDetectionModels, Estimate)
  FrameLabeler               FrameLabeler.h:67-74
  PulseAccumulator           PulseAccumulator.h:68-74

Device buffers are torch CUDA tensors (torch only provides device memory and
the stream); all computation happens in libhw_b200.so.
"""
import ctypes as C

import numpy as np
import torch

from . import abi
from .native import check, lib


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _p(t):
    return None if t is None else C.c_void_p(t.data_ptr())


def struct_buffer(dtype, n, device="cuda"):
    """Uninitialised device buffer for n structs of a numpy structured dtype."""
    return torch.empty(n * dtype.itemsize, dtype=torch.uint8, device=device)


def struct_to_numpy(t, dtype):
    return t.detach().cpu().numpy().view(dtype)


def numpy_to_struct(a, device="cuda"):
    return torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).to(device)


class _Handle:
    _destroy = None

    def __init__(self):
        self._h = C.c_void_p()

    def close(self):
        if self._h and self._h.value:
            getattr(lib(), self._destroy)(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Baseliner(_Handle):
    _destroy = "hw_baseliner_destroy"

    def __init__(self, cfg, pool_id, lanes, frames_per_chunk):
        super().__init__()
        self.lanes, self.F = lanes, frames_per_chunk
        check(lib().hw_baseliner_create(C.byref(cfg), pool_id, lanes, frames_per_chunk, C.byref(self._h)))

    def startup_latency(self):
        v = C.c_uint32()
        check(lib().hw_baseliner_startup_latency(self._h, C.byref(v)))
        return v.value

    def __call__(self, trace, first_frame, out=None, stats=None):
        """Returns (baseline-subtracted traces, per-lane BaselinerStatAccumState).
        `trace` is int16 or uint8 (the two PacketLayout encodings)."""
        assert trace.dtype in (torch.int16, torch.uint8) and trace.is_cuda and trace.is_contiguous()
        out = torch.empty(trace.shape, dtype=torch.int16, device=trace.device) if out is None else out
        stats = struct_buffer(abi.BLSTATS_DT, self.lanes) if stats is None else stats
        fn = lib().hw_baseliner_process_u8 if trace.dtype == torch.uint8 else lib().hw_baseliner_process
        check(fn(self._h, _p(trace), int(first_frame), _p(out), _p(stats), _stream()))
        return out, stats


class BaselineStatsAggregator(_Handle):
    _destroy = "hw_blstats_aggregator_destroy"

    def __init__(self, pool_id, lanes):
        super().__init__()
        self.lanes = lanes
        check(lib().hw_blstats_aggregator_create(pool_id, lanes, C.byref(self._h)))

    def add_metrics(self, stats, frame_interval):
        check(lib().hw_blstats_aggregator_add(self._h, _p(stats), abi.FrameInterval(*frame_interval), _stream()))

    def trace_stats(self):
        out = struct_buffer(abi.BLSTATS_DT, self.lanes)
        fi = abi.FrameInterval()
        check(lib().hw_blstats_aggregator_get(self._h, _p(out), C.byref(fi), _stream()))
        return out, fi.tuple()

    def reset(self):
        check(lib().hw_blstats_aggregator_reset(self._h, _stream()))


class TraceHistogramAccumulator(_Handle):
    _destroy = "hw_histogram_destroy"

    def __init__(self, cfg, pool_id, lanes):
        super().__init__()
        self.lanes = lanes
        check(lib().hw_histogram_create(C.byref(cfg), pool_id, lanes, C.byref(self._h)))

    def add_batch(self, traces, frame_interval, models):
        frames = traces.shape[1]
        check(lib().hw_histogram_add_batch(self._h, _p(traces), frames, abi.FrameInterval(*frame_interval),
                                           _p(models), _stream()))

    def reset_from_stats(self, stats):
        check(lib().hw_histogram_reset_from_stats(self._h, _p(stats), _stream()))

    def reset_from_bounds(self, bounds):
        check(lib().hw_histogram_reset_from_bounds(self._h, _p(bounds), _stream()))

    def histogram(self):
        out = struct_buffer(abi.LANE_HIST_DT, self.lanes)
        fi = abi.FrameInterval()
        check(lib().hw_histogram_get(self._h, _p(out), C.byref(fi), _stream()))
        return out, fi.tuple()


class DmeEmEstimator(_Handle):
    _destroy = "hw_dme_destroy"

    def __init__(self, cfg, pool_id, lanes):
        super().__init__()
        self.lanes = lanes
        check(lib().hw_dme_create(C.byref(cfg), pool_id, lanes, C.byref(self._h)))

    def init_detection_models(self, stats, models=None):
        models = struct_buffer(abi.LANE_MODEL_DT, self.lanes) if models is None else models
        check(lib().hw_dme_init_models(self._h, _p(stats), _p(models), _stream()))
        return models

    def estimate(self, hist, hist_fi, stats, models, model_fi, diag=True):
        """Updates `models` in place; returns per-lane hw_dme_diag (device) or None."""
        d = struct_buffer(abi.DME_DIAG_DT, self.lanes) if diag else None
        check(lib().hw_dme_estimate(self._h, _p(hist), _p(stats), abi.FrameInterval(*hist_fi),
                                    abi.FrameInterval(*model_fi), _p(models), _p(d), _stream()))
        return d

    def estimate_proposal(self, hist, hist_fi, stats, models, model_fi, proposal, diag=True):
        """estimate() from a learned start [lanes][15][64] (hw_dme_estimate_proposal)."""
        d = struct_buffer(abi.DME_DIAG_DT, self.lanes) if diag else None
        check(lib().hw_dme_estimate_proposal(self._h, _p(hist), _p(stats), abi.FrameInterval(*hist_fi),
                                             abi.FrameInterval(*model_fi), _p(models), _p(d), _p(proposal),
                                             _stream()))
        return d

    def profile_phases(self, enable=True):
        check(lib().hw_dme_profile_phases(self._h, 1 if enable else 0))

    def phase_cycles(self):
        """[lanes][8] int64 per-lane phase clock of the last estimate (see
        hw_dme_profile_phases)."""
        out = np.zeros((self.lanes, 8), np.int64)
        check(lib().hw_dme_phase_cycles(self._h, abi.ptr(out), _stream()))
        return out


def em_fit(cfg, lanes, hist, stats, hist_fi, model_fi, models, start=0, proposal=None, target=None, tol=1e-4,
           max_iter=20, scratch=None, at_stop=False):
    """Single-ZMW EM fit (hw_dme_em_fit) on device buffers; returns
    (params [lanes][15][64] float32, iters [lanes][5][64] int32,
    loglike [lanes][3][64] float32) as CUDA tensors, and with at_stop=True
    also the parameters at the first converged iteration [lanes][15][64]."""
    dev = "cuda"
    params = torch.empty((lanes, 15, abi.LANE), dtype=torch.float32, device=dev)
    stop = torch.empty((lanes, 15, abi.LANE), dtype=torch.float32, device=dev) if at_stop else None
    iters = torch.empty((lanes, 5, abi.LANE), dtype=torch.int32, device=dev)
    ll = torch.empty((lanes, 3, abi.LANE), dtype=torch.float32, device=dev)
    if scratch is None:
        nbytes = C.c_uint64()
        check(lib().hw_dme_em_fit_scratch_bytes(lanes, C.byref(nbytes)))
        scratch = torch.empty(nbytes.value // 4, dtype=torch.float32, device=dev)
    check(lib().hw_dme_em_fit(C.byref(cfg), lanes, _p(hist), _p(stats), abi.FrameInterval(*hist_fi),
                              abi.FrameInterval(*model_fi), _p(models), int(start), _p(proposal), _p(target),
                              float(tol), int(max_iter), _p(scratch), _p(params), _p(iters), _p(ll), _p(stop),
                              _stream()))
    return (params, iters, ll, stop) if at_stop else (params, iters, ll)


class FrameLabeler(_Handle):
    _destroy = "hw_labeler_destroy"

    def __init__(self, cfg, pool_id, lanes, frames_per_chunk):
        super().__init__()
        self.lanes, self.F = lanes, frames_per_chunk
        self.latent_frames = lib().hw_labeler_latent_frames()
        check(lib().hw_labeler_create(C.byref(cfg), pool_id, lanes, frames_per_chunk, C.byref(self._h)))

    def __call__(self, traces, models, margin=False):
        """Returns (labels [lanes,F,64] lagging 24 frames, latent traces [lanes,24,64], viterbi score), and
        with margin=True also each label's best-path decision margin [lanes,F,64] (see hw_labeler_process)."""
        labels = torch.empty_like(traces)
        lat = torch.empty((self.lanes, self.latent_frames, abi.LANE), dtype=torch.int16, device=traces.device)
        score = torch.empty((self.lanes, abi.LANE), dtype=torch.float32, device=traces.device)
        mg = torch.empty(traces.shape, dtype=torch.float32, device=traces.device) if margin else None
        check(lib().hw_labeler_process(self._h, _p(traces), _p(models), _p(labels), _p(lat), _p(score),
                                       _p(mg) if margin else None, _stream()))
        return (labels, lat, score, mg) if margin else (labels, lat, score)


class PulseAccumulator(_Handle):
    _destroy = "hw_pulse_accumulator_destroy"

    def __init__(self, cfg, pool_id, lanes, frames_per_chunk):
        super().__init__()
        self.lanes, self.F = lanes, frames_per_chunk
        self.cap = cfg.max_calls_per_zmw
        check(lib().hw_pulse_accumulator_create(C.byref(cfg), pool_id, lanes, frames_per_chunk, C.byref(self._h)))

    def __call__(self, labels, latent, traces, first_frame, models):
        dev = labels.device
        pulses = torch.empty(self.lanes * abi.LANE * self.cap * abi.PULSE_DT.itemsize, dtype=torch.uint8, device=dev)
        lens = torch.empty((self.lanes, abi.LANE), dtype=torch.int32, device=dev)
        ovf = torch.empty((self.lanes, abi.LANE), dtype=torch.int32, device=dev)
        bls = struct_buffer(abi.STAT_ACCUM_DT, self.lanes)
        check(lib().hw_pulse_accumulator_process(self._h, _p(labels), _p(latent), _p(traces), int(first_frame),
                                                 _p(models), _p(pulses), _p(lens), _p(ovf), _p(bls), _stream()))
        return pulses, lens, ovf, bls


class BatchAnalyzer(_Handle):
    """One pool's full chain (BatchAnalyzer + DetectionModelEstimator)."""
    _destroy = "hw_analyzer_destroy"

    def __init__(self, cfg, pool_id, lanes, frames_per_chunk):
        super().__init__()
        self.lanes, self.F = lanes, frames_per_chunk
        self.cap = cfg.max_calls_per_zmw
        check(lib().hw_analyzer_create(C.byref(cfg), pool_id, lanes, frames_per_chunk, C.byref(self._h)))
        dev = "cuda"
        self.pulses = torch.empty(lanes * abi.LANE * self.cap * abi.PULSE_DT.itemsize, dtype=torch.uint8, device=dev)
        self.lens = torch.empty((lanes, abi.LANE), dtype=torch.int32, device=dev)
        self.ovf = torch.empty((lanes, abi.LANE), dtype=torch.int32, device=dev)

    def __call__(self, trace, first_frame, pulses=None, lens=None, ovf=None):
        """Returns (pulses, lens, overflows, emitted, estimated); buffers are reused between calls."""
        pulses = self.pulses if pulses is None else pulses
        lens = self.lens if lens is None else lens
        ovf = self.ovf if ovf is None else ovf
        em, est = C.c_int32(), C.c_int32()
        fn = lib().hw_analyzer_process_u8 if trace.dtype == torch.uint8 else lib().hw_analyzer_process
        check(fn(self._h, _p(trace), int(first_frame), _p(pulses), _p(lens), _p(ovf), C.byref(em), C.byref(est),
                 _stream()))
        return pulses, lens, ovf, bool(em.value), bool(est.value)

    STAGES = ("baseline", "aggregate", "histogram", "model_init", "dme", "hist_reset", "labeler", "pulses", "metrics")

    def export_state(self):
        """Checkpoint of the pool's state as a numpy uint8 array."""
        n = C.c_uint64()
        check(lib().hw_analyzer_state_size(self._h, C.byref(n)))
        blob = np.empty(n.value, np.uint8)
        check(lib().hw_analyzer_state_export(self._h, abi.ptr(blob), n.value, _stream()))
        return blob

    def import_state(self, blob):
        blob = np.ascontiguousarray(blob, np.uint8)
        check(lib().hw_analyzer_state_import(self._h, abi.ptr(blob), blob.size, _stream()))

    def set_learned_init(self, net):
        """Start every estimate from `net`'s proposal (a learned_init.Network,
        kept alive by the caller); None restores the reference start."""
        check(lib().hw_analyzer_set_learned_init(self._h, None if net is None else net._h))
        self._net = net

    def profile(self, enable=True):
        check(lib().hw_analyzer_profile(self._h, 1 if enable else 0))

    def stage_times(self):
        """{stage: (device ms, launches)} since the previous call (synchronises)."""
        import numpy as _np
        ms = _np.zeros(len(self.STAGES), _np.float64)
        n = _np.zeros(len(self.STAGES), _np.uint32)
        check(lib().hw_analyzer_stage_times(self._h, abi.ptr(ms), abi.ptr(n)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.STAGES)}

    def models(self):
        out = struct_buffer(abi.LANE_MODEL_DT, self.lanes)
        fi = abi.FrameInterval()
        check(lib().hw_analyzer_models(self._h, _p(out), C.byref(fi), _stream()))
        return out, fi.tuple()

    def chunk_metrics(self):
        """(baseliner stats, Viterbi scores [lanes][64], pulse-detector baseline
        stats) of the last chunk, as device buffers."""
        bs = struct_buffer(abi.BLSTATS_DT, self.lanes)
        vs = torch.empty((self.lanes, abi.LANE), dtype=torch.float32, device="cuda")
        pd = struct_buffer(abi.STAT_ACCUM_DT, self.lanes)
        check(lib().hw_analyzer_chunk_metrics(self._h, _p(bs), _p(vs), _p(pd), _stream()))
        return bs, vs, pd

    def last_diag(self):
        out = struct_buffer(abi.DME_DIAG_DT, self.lanes)
        valid = C.c_int32()
        check(lib().hw_analyzer_last_diag(self._h, _p(out), C.byref(valid), _stream()))
        return out if valid.value else None


class TraceGenerator(_Handle):
    """Device synthetic-trace source (workload 0, 1, 2 or 4 defaults)."""
    _destroy = "hw_trace_generator_destroy"

    def __init__(self, lanes, workload=1, zmw_offset=0, params=None, seed=None):
        super().__init__()
        self.lanes = lanes
        p = abi.GenParams()
        if params is None:
            check(lib().hw_gen_params_default(int(workload), C.byref(p)))
        else:
            p = params
        if seed is not None:
            p.seed = seed
        self.params = p
        check(lib().hw_trace_generator_create(C.byref(p), lanes, zmw_offset, C.byref(self._h)))

    def next(self, first_frame, frames, out=None):
        out = torch.empty((self.lanes, frames, abi.LANE), dtype=torch.int16, device="cuda") if out is None else out
        check(lib().hw_trace_generator_next(self._h, _p(out), int(first_frame), frames, _stream()))
        return out


def default_config():
    cfg = abi.Config()
    check(lib().hw_config_default(C.byref(cfg)))
    return cfg


class PoolSet(_Handle):
    """Uneven pools in shared launches (hw_pool_set): pools with equal chunk
    length and stagger class run as one batched analyzer."""
    _destroy = "hw_pool_set_destroy"

    def __init__(self, cfg, lanes, frames_per_chunk):
        super().__init__()
        n = len(lanes)
        self.lanes = np.ascontiguousarray(lanes, np.uint32)
        self.frames = np.ascontiguousarray(frames_per_chunk, np.uint32)
        self.cap = cfg.max_calls_per_zmw
        check(lib().hw_pool_set_create(C.byref(cfg), n, abi.ptr(self.lanes), abi.ptr(self.frames), C.byref(self._h)))
        self.offsets = np.zeros(n, np.uint64)
        total = C.c_uint64()
        groups = C.c_uint32()
        check(lib().hw_pool_set_layout(self._h, abi.ptr(self.offsets), C.byref(total), C.byref(groups)))
        self.total, self.launch_groups = total.value, groups.value
        self.packed = torch.empty(self.total, dtype=torch.int16, device="cuda")

    def chunk(self, p):
        """View of pool p's chunk [lanes][F][64] inside the packed input."""
        o, L, F = int(self.offsets[p]), int(self.lanes[p]), int(self.frames[p])
        return self.packed[o:o + L * F * abi.LANE].view(L, F, abi.LANE)

    def process(self, step):
        n = len(self.lanes)
        em = np.zeros(n, np.int32)
        est = np.zeros(n, np.int32)
        check(lib().hw_pool_set_process(self._h, _p(self.packed), int(step), abi.ptr(em), abi.ptr(est), _stream()))
        return em, est

    def outputs(self, p):
        """(pulses, lens, overflows) of pool p: CUDA tensors viewing the set's
        buffers, overwritten by the next step."""
        pp, pl, po = C.c_void_p(), C.c_void_p(), C.c_void_p()
        check(lib().hw_pool_set_outputs(self._h, p, C.byref(pp), C.byref(pl), C.byref(po)))
        L = int(self.lanes[p])
        n = L * abi.LANE
        lens = _from_device(pl.value, n * 4).view(torch.int32).view(L, abi.LANE)
        ovf = _from_device(po.value, n * 4).view(torch.int32).view(L, abi.LANE)
        pulses = _from_device(pp.value, n * self.cap * abi.PULSE_DT.itemsize)
        return pulses, lens, ovf


class FusedEngine(_Handle):
    """All pools of a basecaller in one handle (hw_chunk_fused): each stage of
    a chunk step is one launch over the lanes of every pool that takes it.
    Pool p's results equal those of BatchAnalyzer(cfg, pool_ids[p], lanes[p],
    frames_per_chunk[p]); its outputs of the last step are in
    outputs(p)."""
    _destroy = "hw_fused_destroy"

    def __init__(self, cfg, lanes, frames_per_chunk, pool_ids=None, graphs=False, tuning=None):
        """tuning: {frames_per_chunk: (fuse_label_pulses, labeler_lanes_per_cta)},
        or "auto" for the autotuner's cached choices on this device."""
        super().__init__()
        self.lanes = np.ascontiguousarray(lanes, np.uint32)
        self.frames = np.ascontiguousarray(frames_per_chunk, np.uint32)
        n = len(self.lanes)
        ids = None if pool_ids is None else np.ascontiguousarray(pool_ids, np.uint32)
        self.cap = cfg.max_calls_per_zmw
        check(lib().hw_fused_create(C.byref(cfg), n, abi.ptr(ids), abi.ptr(self.lanes), abi.ptr(self.frames),
                                    C.byref(self._h)))
        self.pulses, self.lens, self.ovf = [], [], []
        self.table = np.zeros(n, abi.POOL_CHUNK_DT)
        for p, L in enumerate(self.lanes):
            z = int(L) * abi.LANE
            self.pulses.append(torch.empty(z * self.cap * abi.PULSE_DT.itemsize, dtype=torch.uint8, device="cuda"))
            self.lens.append(torch.empty((int(L), abi.LANE), dtype=torch.int32, device="cuda"))
            self.ovf.append(torch.empty((int(L), abi.LANE), dtype=torch.int32, device="cuda"))
            self.table["d_pulses"][p] = self.pulses[p].data_ptr()
            self.table["d_lens"][p] = self.lens[p].data_ptr()
            self.table["d_overflows"][p] = self.ovf[p].data_ptr()
        self.next_frame = np.zeros(n, np.int64)
        if graphs:
            self.use_graphs(True)
        if isinstance(tuning, str) and tuning == "auto":
            from . import autotune
            tuning = autotune.load()
        if tuning:
            self.set_tuning(tuning)

    def use_graphs(self, enable=True):
        check(lib().hw_fused_use_graphs(self._h, 1 if enable else 0))

    def set_overlap(self, mode=1):
        """hw_fused_set_overlap: 0 one stream, 1 (default) the DME beside the
        labeling, 2 also the histogram."""
        check(lib().hw_fused_set_overlap(self._h, int(mode)))

    def set_learned_init(self, net):
        """Start every estimate from `net`'s proposal (a learned_init.Network,
        kept alive by the engine), or the reference start (None)."""
        check(lib().hw_fused_set_learned_init(self._h, None if net is None else net._h))
        self._net = net

    def enable_hf_metrics(self, frames_per_block=4096, frame_rate=100.0, realtime_activity_labels=True, cart=None):
        """Adds the HF metrics filter; pool p's block metrics land in
        self.metrics[p] on steps where metrics_emitted()[p] is set."""
        arrs = [None] * 6
        n, maxh = 0, 0.0
        if cart is not None:
            arrs = [np.ascontiguousarray(cart["children_left"], np.int16),
                    np.ascontiguousarray(cart["children_right"], np.int16),
                    np.ascontiguousarray(cart["feature"], np.int8), np.ascontiguousarray(cart["threshold"], np.float32),
                    np.ascontiguousarray(cart["value"], np.int8), np.ascontiguousarray(cart["hsw_curve"], np.float32)]
            n = len(arrs[0])
            maxh = float(np.asarray(cart["max_acceptable_halfsandwich_rate"]).reshape(-1)[0])
        ptrs = [abi.ptr(a) for a in arrs]
        check(lib().hw_fused_enable_hf_metrics(self._h, frames_per_block, float(frame_rate),
                                               1 if realtime_activity_labels else 0, *ptrs[:5], n, ptrs[5], maxh))
        self.metrics = [struct_buffer(abi.BASECALLING_METRICS_DT, int(L)) for L in self.lanes]
        for p, m in enumerate(self.metrics):
            self.table["d_metrics"][p] = m.data_ptr()

    def metrics_emitted(self):
        return self.table["metrics_emitted"].copy()

    def set_tuning(self, tuning):
        """tuning: {frames_per_chunk: (fuse_label_pulses, labeler_lanes_per_cta)}."""
        t = np.zeros(len(tuning), abi.FUSED_TUNING_DT)
        for i, (F, (fuse, lpc)) in enumerate(sorted(tuning.items())):
            t[i] = (F, fuse, lpc, 0)
        check(lib().hw_fused_set_tuning(self._h, abi.ptr(t), len(t)))

    def process(self, chunks, outputs=None):
        """One step: chunks[p] is pool p's next chunk [lanes][F][64] (int16 or
        uint8 CUDA tensor).  outputs[p] = (pulses, lens, overflows) receives
        pool p's results (default: the engine's own buffers, outputs(p)).
        Returns (emitted, estimated) flags per pool."""
        t = self.table
        for p, c in enumerate(chunks):
            if c.dtype == torch.uint8:
                t["d_trace"][p], t["d_trace8"][p] = 0, c.data_ptr()
            else:
                t["d_trace"][p], t["d_trace8"][p] = c.data_ptr(), 0
        outs = outputs if outputs is not None else [self.outputs(p) for p in range(len(t))]
        for p, (pp, pl, po) in enumerate(outs):
            t["d_pulses"][p], t["d_lens"][p], t["d_overflows"][p] = pp.data_ptr(), pl.data_ptr(), po.data_ptr()
        t["first_frame"] = self.next_frame
        check(lib().hw_chunk_fused(self._h, abi.ptr(t), len(t), _stream()))
        self.next_frame += self.frames
        return t["emitted"].copy(), t["estimated"].copy()

    def finish(self):
        check(lib().hw_fused_finish(self._h, _stream()))

    def outputs(self, p):
        """(pulses, lens, overflows) of pool p's last step."""
        return self.pulses[p], self.lens[p], self.ovf[p]

    def last_diag(self, p):
        """Pool p's DME diagnostics of its latest estimate (None before it)."""
        out = struct_buffer(abi.DME_DIAG_DT, int(self.lanes[p]))
        valid = C.c_int32()
        check(lib().hw_fused_last_diag(self._h, int(p), _p(out), C.byref(valid), _stream()))
        return out if valid.value else None

    def models(self, p):
        out = struct_buffer(abi.LANE_MODEL_DT, int(self.lanes[p]))
        fi = abi.FrameInterval()
        check(lib().hw_fused_models(self._h, p, _p(out), C.byref(fi), _stream()))
        return out, fi.tuple()

    def profile(self, enable=True):
        check(lib().hw_fused_profile(self._h, 1 if enable else 0))

    def stage_times(self):
        """{stage: (device ms, launches)} since the previous call (synchronises)."""
        ms = np.zeros(len(BatchAnalyzer.STAGES), np.float64)
        n = np.zeros(len(BatchAnalyzer.STAGES), np.uint32)
        check(lib().hw_fused_stage_times(self._h, abi.ptr(ms), abi.ptr(n)))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(BatchAnalyzer.STAGES)}

    def last_step(self):
        """(kernel launches, graph launches) of the last step."""
        a, b = C.c_uint32(), C.c_uint32()
        check(lib().hw_fused_last_step(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value


class HfMetrics(_Handle):
    """HFMetricsFilter of one pool (hw_hfmetrics)."""
    _destroy = "hw_hfmetrics_destroy"

    def __init__(self, lanes, frames_per_block=4096, frame_rate=100.0, realtime_activity_labels=True, cart=None):
        super().__init__()
        self.lanes = lanes
        check(lib().hw_hfmetrics_create(lanes, frames_per_block, float(frame_rate),
                                        1 if realtime_activity_labels else 0, C.byref(self._h)))
        self.out = struct_buffer(abi.BASECALLING_METRICS_DT, lanes)
        if cart is not None:
            self.set_cart(cart)

    def set_cart(self, cart):
        # converted copies held in locals until the call returns
        left = np.ascontiguousarray(cart["children_left"], np.int16)
        right = np.ascontiguousarray(cart["children_right"], np.int16)
        feature = np.ascontiguousarray(cart["feature"], np.int8)
        thr = np.ascontiguousarray(cart["threshold"], np.float32)
        value = np.ascontiguousarray(cart["value"], np.int8)
        hsw = np.ascontiguousarray(cart["hsw_curve"], np.float32)
        check(lib().hw_hfmetrics_set_cart(self._h, abi.ptr(left), abi.ptr(right), abi.ptr(feature), abi.ptr(thr),
                                          abi.ptr(value), len(left), abi.ptr(hsw),
                                          float(np.asarray(cart["max_acceptable_halfsandwich_rate"]).reshape(-1)[0])))

    def process(self, pulses, lens, cap, baseliner_stats, models, viterbi, pd_stats, first_frame, frames):
        """One pulse batch (device buffers).  Returns the block's metrics
        (device uint8 buffer of BASECALLING_METRICS_DT records) or None."""
        em = C.c_int32()
        check(lib().hw_hfmetrics_process(self._h, _p(pulses), _p(lens), int(cap), _p(baseliner_stats), _p(models),
                                         _p(viterbi), _p(pd_stats), int(first_frame), int(frames), _p(self.out),
                                         C.byref(em), _stream()))
        return self.out if em.value else None


class Repacker(_Handle):
    """Ingest repacking (hw_repacker): sensor packets of one chunk of frames
    gathered into the pools' TraceBatch chunks."""
    _destroy = "hw_repacker_destroy"

    def __init__(self, num_zmw, lanes_per_pool, frames_per_chunk, encoding="int16"):
        super().__init__()
        self.num_zmw, self.lanes_per_pool, self.F = num_zmw, lanes_per_pool, frames_per_chunk
        self.dtype = torch.int16 if encoding == "int16" else torch.uint8
        check(lib().hw_repacker_create(num_zmw, lanes_per_pool, frames_per_chunk, 0 if encoding == "int16" else 1,
                                       C.byref(self._h)))
        n = C.c_uint32()
        check(lib().hw_repacker_num_pools(self._h, C.byref(n)))
        self.n_pools = n.value
        lanes = num_zmw // abi.LANE
        self.pool_lanes = [min(lanes_per_pool, lanes - p * lanes_per_pool) for p in range(self.n_pools)]

    def new_chunks(self):
        return [torch.zeros((L, self.F, abi.LANE), dtype=self.dtype, device="cuda") for L in self.pool_lanes]

    def __call__(self, packets, packet_data, chunk_first_frame, chunks):
        """packets: numpy SENSOR_PACKET_DT table; packet_data: CUDA uint8
        tensor holding the packets; chunks: per-pool CUDA tensors (written)."""
        packets = np.ascontiguousarray(packets, abi.SENSOR_PACKET_DT)
        ptrs = (C.c_void_p * len(chunks))(*[c.data_ptr() for c in chunks])
        check(lib().hw_repack_chunk(self._h, abi.ptr(packets), len(packets), _p(packet_data), int(chunk_first_frame),
                                    ptrs, _stream()))
        return chunks


def baz_preset(which):
    """(fields, skip_rejects) of a basecaller pulse encoding: abi.BAZ_PRODUCTION
    or abi.BAZ_INTERNAL (PulseGroups.h)."""
    fields = np.zeros(16, abi.BAZ_FIELD_DT)
    n, skip = C.c_uint32(), C.c_int32()
    check(lib().hw_baz_preset(int(which), abi.ptr(fields), C.byref(n), C.byref(skip)))
    return fields[:n.value].copy(), bool(skip.value)


class BazEncoder(_Handle):
    """BAZ pulse encoding (hw_baz_encoder): each chunk's pulses of every ZMW
    become that ZMW's bytes (PrelimHQFilter + PacketBuffer::AddZmw).  The
    start-frame delta state of each ZMW carries over between chunks."""
    _destroy = "hw_baz_encoder_destroy"

    def __init__(self, num_zmw, fields=None, skip_rejects=None, preset=abi.BAZ_PRODUCTION, zmw_stride=1):
        super().__init__()
        if fields is None:
            fields, skip = baz_preset(preset)
            skip_rejects = skip if skip_rejects is None else skip_rejects
        self.fields = np.ascontiguousarray(fields, abi.BAZ_FIELD_DT)
        self.num_zmw = num_zmw
        check(lib().hw_baz_encoder_create(abi.ptr(self.fields), len(self.fields), int(bool(skip_rejects)), num_zmw,
                                          C.byref(self._h)))
        if zmw_stride != 1:
            check(lib().hw_baz_encoder_set_zmw_stride(self._h, zmw_stride))
        self.offsets = torch.zeros(num_zmw + 1, dtype=torch.int64, device="cuda")
        self.events = torch.zeros(num_zmw, dtype=torch.int32, device="cuda")
        self.bytes = torch.empty(0, dtype=torch.uint8, device="cuda")

    def __call__(self, pulses, lens, max_calls):
        """pulses: CUDA buffer of [num_zmw][max_calls] hw_pulse; lens: CUDA
        uint32/int32 counts.  Returns (bytes, offsets): the chunk's bytes (a
        view of the encoder's buffer) and the ZMW offsets [num_zmw + 1]; the
        pulses encoded of each ZMW are in self.events."""
        total = C.c_uint64()
        for _ in range(2):
            rc = lib().hw_baz_encode(self._h, _p(pulses), _p(lens), int(max_calls), _p(self.bytes),
                                     self.bytes.numel(), _p(self.offsets), _p(self.events), C.byref(total),
                                     _stream())
            if rc != abi.HW_ERR_OUT_OF_MEMORY:
                break
            self.bytes = torch.empty(max(total.value, 2 * self.bytes.numel()), dtype=torch.uint8, device="cuda")
        check(rc)
        return self.bytes[:total.value], self.offsets

    def enqueue(self, pulses, lens, max_calls, out, offsets, events=None):
        """hw_baz_encode_async into caller buffers (a CUDA uint8 tensor and an
        int64 tensor of num_zmw + 1); offsets[-1] is the chunk's bytes."""
        check(lib().hw_baz_encode_async(self._h, _p(pulses), _p(lens), int(max_calls), _p(out), out.numel(),
                                        _p(offsets), _p(events), _stream()))

    def result(self):
        """Status of the last finished enqueue (after synchronising): its bytes."""
        total = C.c_uint64()
        check(lib().hw_baz_encode_result(self._h, C.byref(total)))
        return total.value


class _DeviceBytes:
    """Device memory owned by the library, exposed to torch without a copy."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def _from_device(ptr, nbytes):
    """uint8 CUDA tensor viewing nbytes of library-owned device memory at ptr
    (valid while the owning handle lives)."""
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device="cuda")


class PrelimHq(_Handle):
    """Preliminary HQ stage (hw_prelim_hq): BAZ-encodes every chunk, keeps the
    last `lookback` metric blocks on the device and produces one checkpoint a
    metric block (PrelimHQFilterBody with the BazAggregator packet side)."""
    _destroy = "hw_prelim_hq_destroy"

    def __init__(self, num_zmw, preset=abi.BAZ_PRODUCTION, fields=None, skip_rejects=None, chunks_per_block=8,
                 lookback=10, enable=False, throttle=0.10, zmw_stride=1, metrics=False):
        super().__init__()
        if fields is None:
            fields, skip = baz_preset(preset)
            skip_rejects = skip if skip_rejects is None else skip_rejects
        self.fields = np.ascontiguousarray(fields, abi.BAZ_FIELD_DT)
        self.num_zmw = num_zmw
        cfg = np.zeros(1, abi.PRELIM_HQ_CONFIG_DT)
        check(lib().hw_prelim_hq_config_default(abi.ptr(cfg)))
        cfg["chunks_per_block"], cfg["lookback_blocks"] = chunks_per_block, lookback
        cfg["enable_prehq"], cfg["hq_throttle_fraction"], cfg["zmw_stride"] = int(bool(enable)), throttle, zmw_stride
        cfg["metrics"] = int(bool(metrics))
        check(lib().hw_prelim_hq_create(abi.ptr(self.fields), len(self.fields), int(bool(skip_rejects)), num_zmw,
                                        abi.ptr(cfg), C.byref(self._h)))
        self._res = np.zeros(1, abi.BAZ_CHECKPOINT_DT)

    def _checkpoint(self):
        r = self._res[0]
        n = self.num_zmw
        return {"bytes": _from_device(int(r["d_bytes"]), int(r["total_bytes"])) if r["total_bytes"] else
                torch.empty(0, dtype=torch.uint8, device="cuda"),
                "offsets": _from_device(int(r["d_offsets"]), 8 * (n + 1)).view(torch.int64),
                "events": _from_device(int(r["d_events"]), 4 * n).view(torch.int32),
                "hq": _from_device(int(r["d_hq"]), n),
                "num_hq": int(r["num_hq"]), "block": int(r["block"])}

    def process(self, pulses, lens, max_calls, metrics=None, marks=None):
        """One chunk; the block's checkpoint (views of the stage's device
        buffers, valid until the next call) when it ends a metric block."""
        produced = C.c_int32()
        check(lib().hw_prelim_hq_process(self._h, _p(pulses), _p(lens), int(max_calls), _p(metrics), _p(marks),
                                         C.byref(produced), abi.ptr(self._res), _stream()))
        return self._checkpoint() if produced.value else None

    def flush(self):
        produced = C.c_int32()
        check(lib().hw_prelim_hq_flush(self._h, C.byref(produced), abi.ptr(self._res), _stream()))
        return self._checkpoint()

    def activity(self):
        out = torch.empty(self.num_zmw, dtype=torch.uint8, device="cuda")
        check(lib().hw_prelim_hq_activity(self._h, _p(out), _stream()))
        return out

    def metric_checkpoint(self):
        """The metric side of the last checkpoint (hw_prelim_hq_metrics):
        {"blocks": uint8 CUDA tensor of total * 164 bytes (abi.
        SPIDER_METRIC_BLOCK_DT records), "offsets": int64 [n + 1], "block"}."""
        r = np.zeros(1, abi.METRIC_CHECKPOINT_DT)
        check(lib().hw_prelim_hq_metrics(self._h, abi.ptr(r)))
        r = r[0]
        n, total = self.num_zmw, int(r["total_blocks"])
        size = abi.SPIDER_METRIC_BLOCK_DT.itemsize
        return {"blocks": _from_device(int(r["d_blocks"]), total * size) if total else
                torch.empty(0, dtype=torch.uint8, device="cuda"),
                "offsets": _from_device(int(r["d_offsets"]), 8 * (n + 1)).view(torch.int64),
                "total": total, "block": int(r["block"])}


class PulseCompactor(_Handle):
    """hw_pulses_compact: the valid pulse records packed ZMW after ZMW, for
    the download of a chunk's results."""
    _destroy = "hw_pulse_compactor_destroy"

    def __init__(self, num_zmw):
        super().__init__()
        self.num_zmw = num_zmw
        check(lib().hw_pulse_compactor_create(num_zmw, C.byref(self._h)))

    def __call__(self, pulses, lens, max_calls, out, offsets):
        """Enqueues the packing into out (CUDA uint8 tensor of num_zmw x
        max_calls records) and offsets (int64, num_zmw + 1); returns the
        mapped slot that will hold the total."""
        slot = C.c_uint32()
        check(lib().hw_pulses_compact(self._h, _p(pulses), _p(lens), int(max_calls), _p(out), _p(offsets),
                                      C.byref(slot), _stream()))
        return slot.value

    def total(self, slot):
        """Records packed by the call that used `slot` (once the stream passed it)."""
        t = C.c_uint64()
        check(lib().hw_pulse_compactor_total(self._h, int(slot), C.byref(t)))
        return t.value
