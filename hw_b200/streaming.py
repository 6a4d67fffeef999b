"""Streaming run: 2,097,152 ZMWs (32,768 lanes in 8 pools)
x 128 chunks of 512 frames, traces generated on the GPU chunk by chunk
(workload 4: 20% amplitude decay over the run, +15 DN baseline step in 1% of
ZMWs at frame 32,768, which the dynamic estimation has to follow), reference
default analysis parameters with dynamic estimation.

The run is made twice, with the reference EM start and with the learned
start (hw_analyzer_set_learned_init), and reports for each the sustained
analysis throughput (device time of the analyzer calls, CUDA events on the
analysis stream, generation excluded and reported apart), the real-time
factor at 100 frames/s and the EM lane iterations per estimate; on one
stream also the per-stage and DME times.  With --streams N the pools'
analyzers run at once on N streams.  The reference host path's rate on this
box's cores is the `cpu_baseline` of bench.py (same analysis parameters).

    python -m hw_b200.streaming [--lanes-per-pool 4096] [--pools 8] [--chunks 128] [--streams 4]
"""
import argparse
import json
import os

import numpy as np
import torch

from . import abi, filters as Fl, workloads

FRAMES = 512
FRAME_RATE = 100.0


def run_chain(cfg, pools, lpp, chunks, net=None, streams=1, engine="analyzers"):
    """One streaming run.  With streams > 1 the pools' analyzers are dealt
    round-robin over that many streams (each with its own copy of the
    learned start's network: a network handle holds its forward pass's
    scratch) and run at once; the stage timers, which time the stream they
    run on, stay off, and only the DME's total is taken from its diagnostics
    (lane iterations).  With one stream every stage is timed.  engine:
    "analyzers" (one hw_analyzer per pool) or "fused" (one one-pool
    hw_chunk_fused engine per pool)."""
    from . import learned_init
    total = pools * lpp
    gen = Fl.TraceGenerator(total, workload=4)
    fused = engine == "fused"
    analyzers = ([Fl.FusedEngine(cfg, [lpp], [FRAMES], pool_ids=[p]) for p in range(pools)] if fused
                 else [Fl.BatchAnalyzer(cfg, p, lpp, FRAMES) for p in range(pools)])
    stream = torch.cuda.current_stream()
    S = max(1, min(streams, pools))
    side = [torch.cuda.Stream() for _ in range(S - 1)]
    nets = []
    if net is not None:
        nets = [net]
        for _ in range(S - 1):
            n = learned_init.Network(max_batch=net.max_batch)
            n.set(*net.get())
            nets.append(n)
    for p, a in enumerate(analyzers):
        if net is not None:
            a.set_learned_init(nets[p % S])
        a.profile(S == 1)
    buf = torch.empty((total, FRAMES, abi.LANE), dtype=torch.int16, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    gen_ms = ana_ms = 0.0
    lane_iters, estimates, emitted = [], 0, 0
    for c in range(chunks):
        ev[0].record(stream)
        gen.next(c * FRAMES, FRAMES, out=buf)
        ev[1].record(stream)
        for s_ in side:
            s_.wait_stream(stream)
        flags = []
        for p, a in enumerate(analyzers):
            with torch.cuda.stream(stream if p % S == 0 else side[p % S - 1]):
                if fused:
                    em, est = a.process([buf[p * lpp:(p + 1) * lpp]])
                    flags.append((None, None, None, bool(em[0]), bool(est[0])))
                else:
                    flags.append(a(buf[p * lpp:(p + 1) * lpp], c * FRAMES))
        for s_ in side:
            stream.wait_stream(s_)
        ev[2].record(stream)
        ev[2].synchronize()
        gen_ms += ev[0].elapsed_time(ev[1])
        ana_ms += ev[1].elapsed_time(ev[2])
        for a, (_, _, _, em, est) in zip(analyzers, flags):
            emitted += int(em)
            if est:
                estimates += 1
                d = Fl.struct_to_numpy(a.last_diag(0) if fused else a.last_diag(), abi.DME_DIAG_DT)
                lane_iters.append(d["lane_iterations"].astype(np.float64))
    stage = {}
    for a in analyzers:
        if S == 1:
            for k, (t, n) in a.stage_times().items():
                s = stage.setdefault(k, [0.0, 0])
                s[0] += t
                s[1] += n
        if fused:
            a.finish()
        a.close()
    for n in nets[1:]:
        n.close()
    gen.close()
    zf = total * abi.LANE * FRAMES * chunks
    rate = zf / (ana_ms / 1e3)
    it = np.concatenate(lane_iters) if lane_iters else np.zeros(1)
    out = {
        "zmw_frames_per_s": rate,
        "real_time_factor": rate / (total * abi.LANE * FRAME_RATE),
        "analysis_ms_per_chunk": ana_ms / chunks,
        "generation_ms_per_chunk": gen_ms / chunks,
        "streams": S,
        "engine": engine,
        "estimates": estimates,
        "em_lane_iterations_mean": float(it.mean()),
        "emitting_pool_chunks": emitted,
    }
    if S == 1:
        out["dme_ms_total"] = stage.get("dme", (0.0, 0))[0]
        out["stage_ms_per_chunk"] = {k: v[0] / chunks for k, v in stage.items()}
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lanes-per-pool", type=int, default=4096)
    ap.add_argument("--pools", type=int, default=8)
    ap.add_argument("--chunks", type=int, default=128)
    ap.add_argument("--weights", default=None, help="trained learned-initializer weights (npz)")
    ap.add_argument("--streams", type=int, default=1, help="streams the pools' analyzers run on")
    ap.add_argument("--engine", choices=["analyzers", "fused"], default="analyzers",
                    help="one hw_analyzer per pool, or one one-pool fused engine per pool")
    a = ap.parse_args()
    from . import learned_init
    cfg = workloads.chip_config()
    net = learned_init.Network()
    if a.weights and os.path.exists(a.weights):
        net.load(a.weights)
    else:
        net, _ = learned_init.run()
        if a.weights:
            net.save(a.weights)
    # inference handle sized for one pool, so each estimate runs one forward pass
    inf = learned_init.Network(max_batch=a.lanes_per_pool * abi.LANE)
    inf.set(*net.get())
    net.close()
    plain = run_chain(cfg, a.pools, a.lanes_per_pool, a.chunks, streams=a.streams, engine=a.engine)
    learned = run_chain(cfg, a.pools, a.lanes_per_pool, a.chunks, inf, streams=a.streams, engine=a.engine)
    out = {"workload": f"streaming: {a.pools * a.lanes_per_pool * abi.LANE} ZMWs x {a.chunks} chunks of {FRAMES} "
                       "frames, generated on the GPU (decay 20%, +15 DN step in 1% of ZMWs), dynamic DME",
           "plain_em": plain, "learned_init": learned}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
