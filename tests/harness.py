"""Drives the oracle and the CUDA filters through the same chunk schedule.

The schedule is the reference's DetectionModelEstimator::AddBatch state
machine (traceAnalysis/DetectionModelEstimator.cpp:93-160) inside the
SingleEstimate / DynamicEstimate batch analyzers (analyzer/BatchAnalyzer.cpp:
172-375).  Both backends see identical inputs at every stage, and every stage
output is recorded so tests can compare them.
"""
import numpy as np

from hw_b200 import abi


class OracleBackend:
    def __init__(self, cfg, lanes, F, pool_id=0):
        import oracle
        self.p = oracle.Pool(cfg, lanes, F, pool_id)
        self.lanes, self.F = lanes, F

    def startup_latency(self):
        return self.p.startup_latency()

    def baseline(self, chunk, ff):
        return self.p.baseline(chunk, ff)

    def agg_add(self, stats, fi):
        self.p.agg_add(stats, fi)

    def agg_get(self):
        return self.p.agg_get()

    def agg_reset(self):
        self.p.agg_reset()

    def hist_reset(self, stats):
        self.p.hist_reset_from_stats(stats)

    def hist_add(self, bls, fi, models):
        self.p.hist_add(bls, fi, models)

    def hist_get(self):
        return self.p.hist_get()

    def init_models(self, stats):
        return self.p.init_models(stats)

    def estimate(self, hist, stats, hfi, mfi, models):
        return self.p.estimate(hist, stats, hfi, mfi, models)

    def label(self, bls, models):
        return self.p.label(bls, models)

    def pulses(self, labels, lat, bls, ff, models):
        return self.p.pulses(labels, lat, bls, ff, models)


class GpuBackend:
    """Same calls on the CUDA filters; inputs/outputs are numpy on the host."""

    def __init__(self, cfg, lanes, F, pool_id=0):
        import torch
        from hw_b200 import filters as Fl
        self.torch, self.Fl = torch, Fl
        self.lanes, self.F = lanes, F
        self.bl = Fl.Baseliner(cfg, pool_id, lanes, F)
        self.agg = Fl.BaselineStatsAggregator(pool_id, lanes)
        self.hist = Fl.TraceHistogramAccumulator(cfg, pool_id, lanes)
        self.dme = Fl.DmeEmEstimator(cfg, pool_id, lanes)
        self.lab = Fl.FrameLabeler(cfg, pool_id, lanes, F)
        self.pa = Fl.PulseAccumulator(cfg, pool_id, lanes, F)
        self.cap = cfg.max_calls_per_zmw

    def _t(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a)).cuda()

    def _s(self, a):
        return self.Fl.numpy_to_struct(a)

    def startup_latency(self):
        return self.bl.startup_latency()

    def baseline(self, chunk, ff):
        out, st = self.bl(self._t(chunk), ff)
        return out.cpu().numpy(), self.Fl.struct_to_numpy(st, abi.BLSTATS_DT)

    def agg_add(self, stats, fi):
        self.agg.add_metrics(self._s(stats), fi)

    def agg_get(self):
        s, fi = self.agg.trace_stats()
        return self.Fl.struct_to_numpy(s, abi.BLSTATS_DT), fi

    def agg_reset(self):
        self.agg.reset()

    def hist_reset(self, stats):
        self.hist.reset_from_stats(self._s(stats))

    def hist_add(self, bls, fi, models):
        self.hist.add_batch(self._t(bls), fi, self._s(models))

    def hist_get(self):
        h, fi = self.hist.histogram()
        return self.Fl.struct_to_numpy(h, abi.LANE_HIST_DT), fi

    def init_models(self, stats):
        return self.Fl.struct_to_numpy(self.dme.init_detection_models(self._s(stats)), abi.LANE_MODEL_DT)

    def estimate(self, hist, stats, hfi, mfi, models):
        m = self._s(models)
        d = self.dme.estimate(self._s(hist), hfi, self._s(stats), m, mfi)
        return self.Fl.struct_to_numpy(m, abi.LANE_MODEL_DT), self.Fl.struct_to_numpy(d, abi.DME_DIAG_DT)

    def label(self, bls, models):
        labels, lat, score = self.lab(self._t(bls), self._s(models))
        return labels.cpu().numpy(), lat.cpu().numpy(), score.cpu().numpy()

    def pulses(self, labels, lat, bls, ff, models):
        p, lens, ovf, b = self.pa(self._t(labels), self._t(lat), self._t(bls), ff, self._s(models))
        pulses = self.Fl.struct_to_numpy(p, abi.PULSE_DT).reshape(self.lanes, abi.LANE, self.cap)
        return pulses, lens.cpu().numpy().astype(np.uint32), ovf.cpu().numpy().astype(np.uint32), \
            self.Fl.struct_to_numpy(b, abi.STAT_ACCUM_DT)


class Pipeline:
    """One pool's analyzer over a backend (FixedModel, SingleEstimate or
    DynamicEstimate)."""

    HIST_INIT, DME_INIT, SEQUENCING = 0, 1, 2

    def __init__(self, backend, cfg, pool_id=0):
        self.b = backend
        self.cfg = cfg
        self.F = backend.F
        self.pool_id = pool_id
        self.status = self.HIST_INIT
        self.frames_remaining = int(cfg.num_frames_pre_accum_stats)
        self.models = None
        self.model_fi = (0, 0)
        self.initialized = False
        self.full_estimation = False
        self.bl_latency = backend.startup_latency()
        F = self.F
        chunks_per_est = (max(int(cfg.min_frames_for_estimate), 1) + F - 1) // F
        self.pool_delay = (pool_id % chunks_per_est) * F

    # DetectionModelEstimator::AddBatch
    def _dme_add(self, bls, stats, fi, rec):
        b = self.b
        b.agg_add(stats, fi)
        if self.status != self.HIST_INIT:
            b.hist_add(bls, fi, self.models)
        if self.status != self.SEQUENCING:
            agg, afi = b.agg_get()
            self.models = b.init_models(agg)
            self.model_fi = afi
            rec["init_models"] = self.models.copy()
        ran = False
        self.frames_remaining -= self.F
        if self.frames_remaining <= 0:
            if self.status == self.DME_INIT:
                self.status = self.SEQUENCING
            if self.status == self.SEQUENCING:
                ran = True
                hist, hfi = b.hist_get()
                agg, afi = b.agg_get()
                rec["hist"] = hist
                rec["agg"] = agg
                self.models, diag = b.estimate(hist, agg, hfi, self.model_fi, self.models)
                self.model_fi = hfi
                rec["models"] = self.models.copy()
                rec["diag"] = diag
            agg, afi = b.agg_get()
            b.hist_reset(agg)
            b.agg_reset()
            if self.status == self.HIST_INIT:
                self.status = self.DME_INIT
            self.frames_remaining = int(self.cfg.min_frames_for_estimate)
        return ran

    def _label_and_pulse(self, bls, ff, rec):
        labels, lat, score = self.b.label(bls, self.models)
        rec["labels"], rec["latent"], rec["score"] = labels, lat, score
        # the labels batch starts LATENT_FRAMES before the trace chunk (LabelsBatch.h:112-121)
        rec["pulses"] = self.b.pulses(labels, lat, bls, ff - abi.LATENT_FRAMES, self.models)

    def process(self, chunk, ff):
        """One chunk; returns the dict of stage outputs."""
        rec = {}
        bls, stats = self.b.baseline(chunk, ff)
        rec["bls"], rec["stats"] = bls, stats
        fi = (ff, ff + self.F)
        mode = self.cfg.model_estimation_mode
        if mode == abi.FIXED_ESTIMATIONS:
            # FixedModelBatchAnalyzer::AnalyzeImpl (BatchAnalyzer.cpp:172-207)
            if self.models is None:
                import oracle
                self.models = oracle.static_model(self.cfg, self.b.lanes)
            self._label_and_pulse(bls, ff, rec)
        elif mode == abi.INITIAL_ESTIMATIONS:
            if not self.initialized and ff > self.bl_latency:
                self.initialized = self._dme_add(bls, stats, fi, rec)
            if self.initialized:
                self._label_and_pulse(bls, ff, rec)
        elif mode == abi.DYNAMIC_ESTIMATIONS:
            if ff < self.bl_latency + self.pool_delay:
                return rec
            if self._dme_add(bls, stats, fi, rec):
                self.full_estimation = True
            self._label_and_pulse(bls, ff, rec)
            rec["emit"] = self.full_estimation
        else:
            raise NotImplementedError("fixed-model analyzer")
        return rec
