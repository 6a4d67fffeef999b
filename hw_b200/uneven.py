"""Uneven pools: 500 pools with lane counts log-uniform in
[1, 2048] and chunk lengths drawn from {128, 256, 512} frames, traces of the
uneven-pool generator (workload 2: per-ZMW lognormal amplitude factors with
sigma 0.3, pulse rates uniform in 0.02-0.12 per frame), reference default
analysis parameters with dynamic estimation.

Ways of running the same pools on the same traces, each timed on its own:
  * fused engine (hw_chunk_fused): every stage of a step is one launch over
    the lanes of all pools that take it; `fused_tuned` with the autotuner's
    kernel choices, `fused_graphs` replaying each step plan as a CUDA graph;
    `fused_streams` deals the pools over four tuned engines that run on four
    streams, so one engine's stages share the GPU with the others';
  * pool set (hw_pool_set): pools that share chunk length and stagger class
    run as one batched analyzer, one launch per stage and class;
  * one analyzer per pool, each with its own launches (what a per-pool
    driver does).
Reported: ZMW-frames/s of the timed steps (device time of the analysis,
CUDA events; trace generation excluded), launches per step.

    python -m hw_b200.uneven [--pools 500] [--steps 4] [--warmup-steps N] [--variants fused,per_pool]
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


def _timed(process, gens, frames, warmup_steps, steps, stream, fill):
    """Runs warmup + timed steps; fill(step) writes every pool's chunk and
    returns the list of chunks; process(step, chunks) enqueues the analysis."""
    t = 0.0
    for step in range(warmup_steps + steps):
        chunks = fill(step)
        ms = _time(lambda: process(step, chunks), stream)
        if step >= warmup_steps:
            t += ms
    return t / steps


def run(n_pools=500, steps=4, warmup_steps=None, variants=("fused_tuned", "fused", "pool_set", "per_pool"), seed=0):
    cfg = workloads.chip_config()
    lanes, frames = pool_shapes(n_pools, seed)
    if warmup_steps is None:
        # every pool past its start-up and in its periodic estimation cycle
        warmup_steps = max(workloads.startup_chunks(cfg, n_pools, int(F)) for F in set(frames.tolist()))
    stream = torch.cuda.current_stream()
    zf_step = int((lanes.astype(np.int64) * frames.astype(np.int64)).sum()) * abi.LANE
    out = {
        "pools": n_pools, "zmws": int(lanes.sum()) * abi.LANE, "lanes_min": int(lanes.min()),
        "lanes_max": int(lanes.max()), "chunk_lengths": sorted(set(int(f) for f in frames)),
        "timed_steps": steps, "warmup_steps": warmup_steps, "zmw_frames_per_step": zf_step,
    }

    def per_pool_buffers():
        return [torch.empty((int(L), int(F), abi.LANE), dtype=torch.int16, device="cuda") for L, F in zip(lanes, frames)]

    for v in variants:
        gens = _gens(lanes)
        if v.startswith("fused"):
            eng = Fl.FusedEngine(cfg, lanes, frames, graphs=(v == "fused_graphs"),
                                 tuning="auto" if v == "fused_tuned" else None)
            bufs = per_pool_buffers()

            def fill(step):
                for p, (g, F) in enumerate(zip(gens, frames)):
                    g.next(step * int(F), int(F), out=bufs[p])
                return bufs
            ms = _timed(lambda step, ch: eng.process(ch), gens, frames, warmup_steps, steps, stream, fill)
            eng.finish()
            out[v + "_launches_per_step"] = list(eng.last_step())
            eng.close()
            del bufs
        elif v == "fused_streams":
            # the pools dealt round-robin over four tuned engines (each keeps
            # its pools' ids), the engines on four streams
            G = 4
            groups = [list(range(g, n_pools, G)) for g in range(G)]
            engs = [Fl.FusedEngine(cfg, lanes[idx], frames[idx], pool_ids=idx, tuning="auto") for idx in groups]
            side = [torch.cuda.Stream() for _ in range(G - 1)]
            bufs = per_pool_buffers()

            def fill(step):
                for p, (g, F) in enumerate(zip(gens, frames)):
                    g.next(step * int(F), int(F), out=bufs[p])
                return bufs

            def on_streams(step, ch):
                for s_ in side:
                    s_.wait_stream(stream)
                for e, idx, s_ in zip(engs, groups, [stream] + side):
                    with torch.cuda.stream(s_):
                        e.process([ch[p] for p in idx])
                for s_ in side:
                    stream.wait_stream(s_)
            ms = _timed(on_streams, gens, frames, warmup_steps, steps, stream, fill)
            last = [e.last_step() for e in engs]
            out[v + "_launches_per_step"] = [sum(x[0] for x in last), sum(x[1] for x in last)]
            for e in engs:
                e.finish()
                e.close()
            del bufs
        elif v == "pool_set":
            ps = Fl.PoolSet(cfg, lanes, frames)

            def fill(step):
                for p, (g, F) in enumerate(zip(gens, frames)):
                    g.next(step * int(F), int(F), out=ps.chunk(p))
                return None
            ms = _timed(lambda step, ch: ps.process(step), gens, frames, warmup_steps, steps, stream, fill)
            out["pool_set_launch_classes"] = ps.launch_groups
            ps.close()
        else:
            ans = [Fl.BatchAnalyzer(cfg, p, int(L), int(F)) for p, (L, F) in enumerate(zip(lanes, frames))]
            bufs = per_pool_buffers()

            def fill(step):
                for p, (g, F) in enumerate(zip(gens, frames)):
                    g.next(step * int(F), int(F), out=bufs[p])
                return bufs

            def one_by_one(step, ch):
                for p, a in enumerate(ans):
                    a(ch[p], step * int(frames[p]))
            ms = _timed(one_by_one, gens, frames, warmup_steps, steps, stream, fill)
            for a in ans:
                a.close()
            del bufs
        for g in gens:
            g.close()
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        out[v + "_ms_per_step"] = ms
        out[v + "_zmw_frames_per_s"] = zf_step / (ms / 1e3)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pools", type=int, default=500)
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--warmup-steps", type=int, default=None)
    ap.add_argument("--variants", default="fused_tuned,fused_streams,fused,pool_set,per_pool")
    a = ap.parse_args()
    print(json.dumps(run(a.pools, a.steps, a.warmup_steps, tuple(a.variants.split(",")))))


if __name__ == "__main__":
    main()
