"""Learned DME initializer: data, training and evaluation on the GPU.

The network (hw_learned_init_* in libhw_b200.so) maps a ZMW's 300-bin trace
histogram and baseline statistics to an EM start; hw_dme_em_fit runs the
reference's EM from it and falls back to the reference's own start whenever
the proposal's log-likelihood is lower.  Nothing here has a counterpart in
the reference.

Data.  Traces come from the uneven-pool generator (workload 2: per-ZMW
lognormal amplitude factors with sigma 0.3, pulse rates uniform in
0.02-0.12 per frame).  Each pool runs the single-estimate schedule of
DetectionModelEstimator (statistics pre-accumulation, then a 4096-frame
histogram) up to its first estimate; the inputs of that estimate (histogram,
baseliner statistics, prior model) are kept.  The label of a ZMW is the
fixed point of the reference's EM from the reference start, run for
`fit_iters` iterations.

Metrics, each from the plain start and from the learned start:
  * iterations to the fixed point: the first iteration whose 15 parameters
    (fractions, means, variances) are all within 1e-4 relative (floors
    0.01 / 1 DN / 1 DN^2) of the plain EM's fixed point;
  * iterations to the parameter-step rule: the first iteration whose update
    changes no parameter by more than 1e-4 relative;
  * iterations to the reference's own stopping rule (log-likelihood gain
    below 1e-4 of |logL|, DmeEmHost.cpp:458-475).
ZMWs whose plain EM does not reach its own fixed point within the budget are
left out of the averages and counted in `resolved_fraction`.
"""
import ctypes as C

import numpy as np
import torch

from . import abi, filters as Fl, workloads
from .native import check, lib

FEAT, OUT, OUT_USED = 304, 32, 19
NORM_SIZE = 2 * FEAT + 2 * OUT


def data_config():
    """Single-estimate schedule with a 4096-frame histogram."""
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.INITIAL_ESTIMATIONS
    cfg.min_frames_for_estimate = 4096
    return cfg


class Pool:
    """The inputs of one pool's first DME estimate, on the device."""

    def __init__(self, cfg, lanes, hist, stats, hist_fi, models, model_fi):
        self.cfg, self.lanes = cfg, lanes
        self.hist, self.stats, self.models = hist, stats, models
        self.hist_fi, self.model_fi = hist_fi, model_fi


def estimate_inputs(cfg, lanes, pool_id=0, seed=None, frames_per_chunk=512, workload=2):
    """Runs the baseliner and the DetectionModelEstimator schedule
    (DetectionModelEstimator.cpp:93-160, single-estimate analyzer) on
    generated traces until the first estimate is due; returns its Pool."""
    F = frames_per_chunk
    gen = Fl.TraceGenerator(lanes, workload=workload, zmw_offset=pool_id * lanes * abi.LANE, seed=seed)
    bl = Fl.Baseliner(cfg, pool_id, lanes, F)
    agg = Fl.BaselineStatsAggregator(pool_id, lanes)
    hist = Fl.TraceHistogramAccumulator(cfg, pool_id, lanes)
    dme = Fl.DmeEmEstimator(cfg, pool_id, lanes)
    HIST_INIT, DME_INIT, SEQUENCING = 0, 1, 2
    status, remaining = HIST_INIT, int(cfg.num_frames_pre_accum_stats)
    latency = bl.startup_latency()
    models = model_fi = None
    trace = torch.empty((lanes, F, abi.LANE), dtype=torch.int16, device="cuda")
    for c in range(100000):
        ff = c * F
        gen.next(ff, F, out=trace)
        bls, st = bl(trace, ff)
        if ff <= latency:
            continue
        fi = (ff, ff + F)
        agg.add_metrics(st, fi)
        if status != HIST_INIT:
            hist.add_batch(bls, fi, models)
        if status != SEQUENCING:
            s, afi = agg.trace_stats()
            models = dme.init_detection_models(s).clone()
            model_fi = afi
        remaining -= F
        if remaining <= 0:
            if status == DME_INIT:
                status = SEQUENCING
            if status == SEQUENCING:
                h, hfi = hist.histogram()
                s, _ = agg.trace_stats()
                out = Pool(cfg, lanes, h.clone(), s.clone(), hfi, models, model_fi)
                for o in (gen, bl, agg, hist, dme):
                    o.close()
                return out
            s, _ = agg.trace_stats()
            hist.reset_from_stats(s)
            agg.reset()
            if status == HIST_INIT:
                status = DME_INIT
            remaining = int(cfg.min_frames_for_estimate)
    raise RuntimeError("estimate never became due")


def fit(pool, start=0, proposal=None, target=None, tol=1e-4, max_iter=1000, at_stop=False):
    """hw_dme_em_fit on a Pool: (params [lanes][15][64], iters [lanes][5][64],
    loglike [lanes][3][64]) CUDA tensors, and with at_stop=True the
    parameters at the first iteration that passes the reference's test."""
    return Fl.em_fit(pool.cfg, pool.lanes, pool.hist, pool.stats, pool.hist_fi, pool.model_fi, pool.models,
                     start=start, proposal=proposal, target=target, tol=tol, max_iter=max_iter, at_stop=at_stop)


def features(pool):
    out = torch.empty((pool.lanes * abi.LANE, FEAT), dtype=torch.float32, device="cuda")
    check(lib().hw_learned_init_features(pool.lanes, Fl._p(pool.hist), Fl._p(pool.stats), Fl._p(out), Fl._stream()))
    return out


def targets(pool, params):
    out = torch.empty((pool.lanes * abi.LANE, OUT), dtype=torch.float32, device="cuda")
    check(lib().hw_learned_init_targets(C.byref(pool.cfg), pool.lanes, Fl._p(params), Fl._p(pool.hist), Fl._p(out),
                                        Fl._stream()))
    return out


class Network:
    """One hw_learned_init handle: BF16 MLP with FP32 master weights and AdamW."""

    def __init__(self, max_batch=4096, seed=1):
        self._h = C.c_void_p()
        check(lib().hw_learned_init_create(max_batch, seed, C.byref(self._h)))
        n = C.c_uint32()
        check(lib().hw_learned_init_param_count(C.byref(n)))
        self.n_params = n.value
        self.max_batch = max_batch

    def close(self):
        if self._h:
            lib().hw_learned_init_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get(self):
        p = np.empty(self.n_params, np.float32)
        nm = np.empty(NORM_SIZE, np.float32)
        check(lib().hw_learned_init_get_params(self._h, abi.ptr(p), abi.ptr(nm)))
        return p, nm

    def set(self, params=None, norm=None):
        p = None if params is None else np.ascontiguousarray(params, np.float32)
        nm = None if norm is None else np.ascontiguousarray(norm, np.float32)
        check(lib().hw_learned_init_set_params(self._h, abi.ptr(p), abi.ptr(nm)))

    def save(self, path):
        p, nm = self.get()
        np.savez(path, params=p, norm=nm)

    def load(self, path):
        d = np.load(path)
        self.set(d["params"], d["norm"])

    def fit_normalization(self, feats, tgts):
        """Input and output standardisation from (up to 262,144 of) the
        training rows, computed on the host."""
        nm = np.zeros(NORM_SIZE, np.float32)
        rows = np.random.default_rng(0).permutation(feats.shape[0])[:262144]
        sel = torch.from_numpy(np.sort(rows)).cuda()
        f = feats.index_select(0, sel).cpu().numpy().astype(np.float64)
        t = tgts.index_select(0, sel).cpu().numpy().astype(np.float64)
        nm[:FEAT] = f.mean(0)
        nm[FEAT:2 * FEAT] = np.maximum(f.std(0), 1e-3)
        nm[2 * FEAT:2 * FEAT + OUT] = t.mean(0)
        nm[2 * FEAT + OUT:] = np.maximum(t.std(0), 1e-4)
        nm[2 * FEAT + OUT_USED:2 * FEAT + OUT] = 0.0
        nm[2 * FEAT + OUT + OUT_USED:] = 1.0
        self.set(norm=nm)

    def forward(self, feats):
        out = torch.empty((feats.shape[0], OUT), dtype=torch.float32, device="cuda")
        check(lib().hw_learned_init_forward(self._h, Fl._p(feats), feats.shape[0], Fl._p(out), Fl._stream()))
        return out

    def forward_status(self):
        """Raises if a forward pass since the last call gave up a bounded
        tensor-core wait (its rows are NaN)."""
        check(lib().hw_learned_init_forward_status(self._h))

    def propose(self, pool):
        """Features, forward pass and EM start in one launch
        (hw_learned_init_propose); equals proposal(pool, forward(features(pool)))."""
        P = torch.empty((pool.lanes, 15, abi.LANE), dtype=torch.float32, device="cuda")
        check(lib().hw_learned_init_propose(self._h, pool.lanes, Fl._p(pool.hist), Fl._p(pool.stats), Fl._p(P),
                                            Fl._stream()))
        return P

    def proposal(self, pool, out):
        P = torch.empty((pool.lanes, 15, abi.LANE), dtype=torch.float32, device="cuda")
        check(lib().hw_learned_init_proposal(self._h, pool.lanes, Fl._p(out), Fl._p(pool.hist), Fl._p(P),
                                             Fl._stream()))
        return P

    def gradients(self, feats, tgts, index=None):
        g = torch.empty(self.n_params, dtype=torch.float32, device="cuda")
        loss = C.c_float()
        n = feats.shape[0] if index is None else index.shape[0]
        check(lib().hw_learned_init_gradients(self._h, Fl._p(feats), Fl._p(tgts), Fl._p(index), n, Fl._p(g),
                                              C.byref(loss), Fl._stream()))
        return loss.value, g

    def train(self, feats, tgts, epochs=20, batch=4096, lr=1e-3, weight_decay=0.01, seed=0, log=None,
              lr_final=1e-5):
        """AdamW over shuffled mini-batches (the shuffle is an index permutation
        drawn on the host; the kernels gather the rows), with the learning
        rate decaying from lr to lr_final on a cosine over all steps."""
        n = feats.shape[0]
        rng = np.random.default_rng(seed)
        loss = C.c_float()
        history = []
        per_epoch = max(n // batch, 1)
        total = epochs * per_epoch
        step = 0
        for ep in range(epochs):
            perm = torch.from_numpy(rng.permutation(n).astype(np.int32)).cuda()
            tot, steps = 0.0, 0
            for i0 in range(0, n - batch + 1, batch):
                idx = perm[i0:i0 + batch]
                lr_t = lr_final + 0.5 * (lr - lr_final) * (1.0 + np.cos(np.pi * step / max(total, 1)))
                step += 1
                check(lib().hw_learned_init_train_step(self._h, Fl._p(feats), Fl._p(tgts), Fl._p(idx), batch, lr_t,
                                                       weight_decay, C.byref(loss), Fl._stream()))
                tot += loss.value
                steps += 1
            history.append(tot / max(steps, 1))
            if log:
                log(f"epoch {ep}: loss {history[-1]:.5f}")
        return history


def _pools(cfg, n_pools, lanes, first_id, seed):
    return [estimate_inputs(cfg, lanes, pool_id=first_id + i, seed=seed) for i in range(n_pools)]


def dataset(pools, fit_iters):
    """Features, targets and plain fixed points of a list of pools."""
    feats, tgts, fixed = [], [], []
    for p in pools:
        params, _, _ = fit(p, start=0, max_iter=fit_iters)
        feats.append(features(p))
        tgts.append(targets(p, params))
        fixed.append(params)
    return torch.cat(feats), torch.cat(tgts), fixed


def param_distance(a, b):
    """Largest relative distance over the 15 EM parameters of each ZMW
    ([lanes][15][64] arrays), floors 0.01 / 1 DN / 1 DN^2 as in hw_dme_em_fit."""
    floor = np.array([0.01] * 5 + [1.0] * 10, np.float32)[None, :, None]
    return (np.abs(a - b) / np.maximum(np.abs(b), floor)).max(1)


def evaluate(net, pools, fixed, fit_iters, tol=1e-4, settle=100):
    """EM iterations to the plain fixed point at `tol`, from the plain and the
    learned start (with fallback), on pools not used for training.  A ZMW is
    resolved when its plain EM comes within tol of its own fixed point at
    least `settle` iterations before the end of the budget."""
    plain_it, learned_it, fell, final_ok, conv_plain, conv_learned, resolved_all = [], [], [], [], [], [], []
    step_plain, step_learned = [], []
    both_conv, stop_agree, stop_plain_fixed, stop_learned_fixed = [], [], [], []
    for p, tgt in zip(pools, fixed):
        _, ip, _, sp = fit(p, start=0, target=tgt, tol=tol, max_iter=fit_iters, at_stop=True)
        out = net.forward(features(p))
        prop = net.proposal(p, out)
        pl, il, _, sl = fit(p, start=abi.EM_START_BETTER, proposal=prop, target=tgt, tol=tol, max_iter=fit_iters,
                            at_stop=True)
        ip, il = ip.cpu().numpy(), il.cpu().numpy()
        # the reference's stopping rule: iterations to it from either start,
        # and how close the estimates kept there are to each other and to
        # the plain fixed point
        sp, sl, tg = sp.cpu().numpy(), sl.cpu().numpy(), tgt.cpu().numpy()
        both = (ip[:, 0] >= 0) & (il[:, 0] >= 0)
        both_conv.append(both.ravel())
        stop_agree.append((param_distance(sl, sp) <= tol)[both])
        stop_plain_fixed.append((param_distance(sp, tg) <= tol)[both])
        stop_learned_fixed.append((param_distance(sl, tg) <= tol)[both])
        res = (ip[:, 1] >= 0) & (ip[:, 1] <= fit_iters - settle)
        resolved_all.append(res.ravel())
        plain_it.append(ip[:, 1][res])
        learned_it.append(np.where(il[:, 1] < 0, fit_iters, il[:, 1])[res])
        fell.append(il[:, 2].ravel())
        final_ok.append((param_distance(pl.cpu().numpy(), tgt.cpu().numpy()) <= tol)[res])
        conv_plain.append(ip[:, 0][ip[:, 0] >= 0])
        conv_learned.append(il[:, 0][il[:, 0] >= 0])
        step_plain.append(np.where(ip[:, 4] < 0, fit_iters, ip[:, 4])[res])
        step_learned.append(np.where(il[:, 4] < 0, fit_iters, il[:, 4])[res])
    cat = np.concatenate
    pi, li = cat(plain_it).astype(np.float64), cat(learned_it).astype(np.float64)
    return {
        "zmws": int(cat(resolved_all).size),
        "resolved_fraction": float(cat(resolved_all).mean()),
        "em_iters_plain_mean": float(pi.mean()),
        "em_iters_learned_mean": float(li.mean()),
        "em_iters_ratio": float(pi.mean() / max(li.mean(), 1e-9)),
        "fallback_rate": float(cat(fell).mean()),
        "final_within_tol_fraction": float(cat(final_ok).mean()),
        "tol": tol,
        "fit_iters": fit_iters,
        "reference_criterion_iters_plain_mean": float(cat(conv_plain).mean()),
        "reference_criterion_iters_learned_mean": float(cat(conv_learned).mean()),
        "step_criterion_iters_plain_mean": float(cat(step_plain).mean()),
        "step_criterion_iters_learned_mean": float(cat(step_learned).mean()),
        # both north-star figures on one criterion at a time
        "criteria": {
            "reference_stopping_rule": {
                "iters_ratio": float(cat(conv_plain).mean() / max(cat(conv_learned).mean(), 1e-9)),
                "within_tol_of_plain_fraction": float(cat(stop_agree).mean()),
                "plain_stop_within_tol_of_fixed_point": float(cat(stop_plain_fixed).mean()),
                "learned_stop_within_tol_of_fixed_point": float(cat(stop_learned_fixed).mean()),
                "zmws_both_converged_fraction": float(cat(both_conv).mean()),
            },
            "distance_to_plain_fixed_point": {
                "iters_ratio": float(pi.mean() / max(li.mean(), 1e-9)),
                "within_tol_of_plain_fraction": float(cat(final_ok).mean()),
                "resolved_fraction": float(cat(resolved_all).mean()),
            },
        },
    }


def dme_phases(net, pool, pool_id=0, sm_mhz=None):
    """Where the DME's time goes, plain start against the learned start, on
    one pool's estimate (the product's lane-wide estimate, hw_dme_estimate /
    hw_dme_estimate_proposal): launch time (CUDA events), the network's own
    time (features, forward pass, proposal columns), lane EM iterations
    (mean, max, share of lanes at the iteration limit) and the per-lane phase
    clock summed over lanes as a share of all lane cycles.  The launch time
    follows the slowest lanes of each SM's lane waves, not the mean."""
    cfg, lanes = pool.cfg, pool.lanes
    names = ["setup", "start_choice", "e_steps", "m_steps", "confidence_blend"]
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

    def one(use_net):
        dme = Fl.DmeEmEstimator(cfg, pool_id, lanes)
        dme.profile_phases(True)
        models = pool.models.clone()
        torch.cuda.synchronize()
        ev[0].record()
        prop = None
        if use_net:
            prop = net.propose(pool)
        ev[1].record()
        if use_net:
            dme.estimate_proposal(pool.hist, pool.hist_fi, pool.stats, models, pool.model_fi, prop, diag=False)
        else:
            dme.estimate(pool.hist, pool.hist_fi, pool.stats, models, pool.model_fi, diag=False)
        ev[2].record()
        ev[2].synchronize()
        ph = dme.phase_cycles()
        dme.close()
        it = ph[:, 5].astype(np.float64)
        tot = ph[:, :5].sum()
        out = {"network_ms": ev[0].elapsed_time(ev[1]), "estimate_ms": ev[1].elapsed_time(ev[2]),
               "lane_iterations_mean": float(it.mean()), "lane_iterations_max": int(it.max()),
               "lanes_at_iteration_limit": float((it >= cfg.em_iteration_limit).mean()),
               "phase_share": {n: float(ph[:, i].sum() / tot) for i, n in enumerate(names)},
               "lane_cycles_mean": float(ph[:, 6].mean()), "lane_cycles_max": int(ph[:, 6].max())}
        if use_net:
            out["zmws_kept_reference_start"] = float(ph[:, 7].sum() / (lanes * abi.LANE))
            out["lanes_with_a_kept_reference_start"] = float((ph[:, 7] > 0).mean())
        # the same estimate without the phase clock (the kernel variant the
        # product runs): its launch time is the stage's
        dme = Fl.DmeEmEstimator(cfg, pool_id, lanes)
        models = pool.models.clone()
        torch.cuda.synchronize()
        ev[2].record()
        if use_net:
            dme.estimate_proposal(pool.hist, pool.hist_fi, pool.stats, models, pool.model_fi, prop, diag=False)
        else:
            dme.estimate(pool.hist, pool.hist_fi, pool.stats, models, pool.model_fi, diag=False)
        ev[3].record()
        ev[3].synchronize()
        dme.close()
        out["estimate_ms_with_clock"] = out["estimate_ms"]
        out["estimate_ms"] = ev[2].elapsed_time(ev[3])
        return out

    one(False), one(True)   # warm-up: module loading and first-launch costs
    return {"lanes": lanes, "plain": one(False), "learned": one(True)}


def run(train_pools=8, eval_pools=1, lanes=4096, fit_iters=1000, epochs=40, batch=4096, lr=1e-3, seed=7, log=None):
    """Generate, label, train and evaluate; returns (network, metrics)."""
    cfg = data_config()
    train = _pools(cfg, train_pools, lanes, 0, seed)
    feats, tgts, _ = dataset(train, fit_iters)
    del train
    net = Network(max_batch=batch, seed=seed)
    net.fit_normalization(feats, tgts)
    history = net.train(feats, tgts, epochs=epochs, batch=batch, lr=lr, seed=seed, log=log)
    del feats, tgts
    held = _pools(cfg, eval_pools, lanes, 1000, seed)
    fixed = [fit(p, start=0, max_iter=fit_iters)[0] for p in held]
    metrics = evaluate(net, held, fixed, fit_iters)
    metrics["dme_phases"] = dme_phases(net, held[0], pool_id=1000)
    metrics["train_zmws"] = train_pools * lanes * abi.LANE
    metrics["final_train_loss"] = history[-1] if history else None
    return net, metrics


def network_timing(lanes=4096, reps=4, seed=1):
    """Device time of the network on lanes * 64 ZMWs (synthetic histograms
    and statistics, a randomly initialised network): the three-step path
    (features, tensor-core forward pass, proposal) and the fused proposal,
    each a launch; the last of `reps` repetitions is reported."""
    rng = np.random.default_rng(seed)
    hist = np.zeros(lanes, abi.LANE_HIST_DT)
    hist["bin_count"] = rng.integers(0, 40, hist["bin_count"].shape)
    hist["low_bound"] = rng.uniform(-50, 0, hist["low_bound"].shape)
    hist["bin_size"] = rng.uniform(0.5, 2, hist["bin_size"].shape)
    st = np.zeros(lanes, abi.BLSTATS_DT)
    st["baseline_stats"]["moment0"] = 1000.0
    st["baseline_stats"]["moment1"] = 3000.0
    st["baseline_stats"]["moment2"] = 30000.0
    pool = Pool(data_config(), lanes, torch.from_numpy(hist.view(np.uint8)).cuda(),
                torch.from_numpy(st.view(np.uint8)).cuda(), None, None, None)
    net = Network(max_batch=4096, seed=seed)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    for _ in range(reps):
        torch.cuda.synchronize()
        ev[0].record()
        f = features(pool)
        ev[1].record()
        y = net.forward(f)
        ev[2].record()
        p3 = net.proposal(pool, y)
        ev[3].record()
        pf = net.propose(pool)
        ev[4].record()
        ev[4].synchronize()
    net.forward_status()
    rows = lanes * abi.LANE
    fwd = ev[1].elapsed_time(ev[2])
    flops = 2.0 * rows * (FEAT * 256 + 256 * 256 + 256 * OUT)
    out = {"rows": rows, "features_ms": ev[0].elapsed_time(ev[1]), "forward_ms": fwd,
           "proposal_ms": ev[2].elapsed_time(ev[3]), "fused_propose_ms": ev[3].elapsed_time(ev[4]),
           "forward_tflops": flops / (fwd / 1e3) / 1e12,
           "fused_equals_three_steps": bool(torch.equal(p3, pf))}
    net.close()
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="train and evaluate the learned DME initializer")
    ap.add_argument("--train-pools", type=int, default=8)
    ap.add_argument("--eval-pools", type=int, default=1)
    ap.add_argument("--lanes", type=int, default=4096)
    ap.add_argument("--fit-iters", type=int, default=1000)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--save", default=None)
    ap.add_argument("--network-timing", action="store_true", help="time the network alone (no training)")
    a = ap.parse_args()
    if a.network_timing:
        print(json.dumps(network_timing(a.lanes)))
        raise SystemExit(0)
    net, m = run(a.train_pools, a.eval_pools, a.lanes, a.fit_iters, a.epochs, log=print)
    if a.save:
        net.save(a.save)
    print(json.dumps(m))
