"""Uneven pools: 500 pools with lane counts log-uniform in
[1, 2048] and chunk lengths drawn from {128, 256, 512} frames, traces of the
uneven-pool generator (workload 2: per-ZMW lognormal amplitude factors with
sigma 0.3, pulse rates uniform in 0.02-0.12 per frame), reference default
analysis parameters with dynamic estimation.

Two ways of running the same pools on the same traces are timed:
  * pool set (hw_pool_set): pools that share chunk length and stagger class
    run as one batched analyzer, one launch per stage and class;
  * one analyzer per pool, each with its own launches (what a per-pool
    driver does).
Reported: ZMW-frames/s of the timed steps (device time of the analysis,
CUDA events; trace generation excluded) and the number of launch classes.

    python -m hw_b200.uneven [--pools 500] [--steps 4] [--warmup-steps N]
"""
import argparse
import json

import numpy as np
import torch

from . import abi, filters as Fl, workloads


def pool_shapes(n_pools, seed=0):
    rng = np.random.default_rng(seed)
    lanes = np.floor(np.exp(rng.uniform(0.0, np.log(2049.0), n_pools))).astype(np.uint32)
    lanes = np.clip(lanes, 1, 2048)
    frames = rng.choice(np.array([128, 256, 512], np.uint32), n_pools)
    return lanes, frames


def _time(fn, stream):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fn()
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1)


def _gens(lanes):
    return [Fl.TraceGenerator(int(L), workload=2, zmw_offset=int(lanes[:p].sum()) * abi.LANE)
            for p, L in enumerate(lanes)]


def run(n_pools=500, steps=4, warmup_steps=None, per_pool=True, seed=0):
    cfg = workloads.chip_config()
    lanes, frames = pool_shapes(n_pools, seed)
    if warmup_steps is None:
        # every pool past its start-up and in its periodic estimation cycle
        warmup_steps = max(workloads.startup_chunks(cfg, n_pools, int(F)) for F in set(frames.tolist()))
    stream = torch.cuda.current_stream()
    zf_step = int((lanes.astype(np.int64) * frames.astype(np.int64)).sum()) * abi.LANE

    # pool set: one launch per stage and schedule class
    ps = Fl.PoolSet(cfg, lanes, frames)
    gens = _gens(lanes)
    t_set = 0.0
    for step in range(warmup_steps + steps):
        for p, (g, F) in enumerate(zip(gens, frames)):
            g.next(step * int(F), int(F), out=ps.chunk(p))
        ms = _time(lambda: ps.process(step), stream)
        if step >= warmup_steps:
            t_set += ms
    classes = ps.launch_groups
    ps.close()
    for g in gens:
        g.close()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    out = {
        "pools": n_pools, "zmws": int(lanes.sum()) * abi.LANE, "lanes_min": int(lanes.min()),
        "lanes_max": int(lanes.max()), "chunk_lengths": sorted(set(int(f) for f in frames)),
        "launch_classes": classes, "timed_steps": steps, "warmup_steps": warmup_steps,
        "zmw_frames_per_step": zf_step,
        "pool_set_zmw_frames_per_s": zf_step * steps / (t_set / 1e3),
        "pool_set_ms_per_step": t_set / steps,
    }
    if not per_pool:
        return out

    # one analyzer per pool on the same traces
    ans = [Fl.BatchAnalyzer(cfg, p, int(L), int(F)) for p, (L, F) in enumerate(zip(lanes, frames))]
    gens = _gens(lanes)
    bufs = [torch.empty((int(L), int(F), abi.LANE), dtype=torch.int16, device="cuda") for L, F in zip(lanes, frames)]
    t_pool = 0.0
    for step in range(warmup_steps + steps):
        for p, (g, F) in enumerate(zip(gens, frames)):
            g.next(step * int(F), int(F), out=bufs[p])

        def one_by_one():
            for p, a in enumerate(ans):
                a(bufs[p], step * int(frames[p]))
        ms = _time(one_by_one, stream)
        if step >= warmup_steps:
            t_pool += ms
    for a in ans:
        a.close()
    out["per_pool_zmw_frames_per_s"] = zf_step * steps / (t_pool / 1e3)
    out["per_pool_ms_per_step"] = t_pool / steps
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pools", type=int, default=500)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup-steps", type=int, default=None)
    ap.add_argument("--no-per-pool", action="store_true")
    a = ap.parse_args()
    print(json.dumps(run(a.pools, a.steps, a.warmup_steps, not a.no_per_pool)))


if __name__ == "__main__":
    main()
