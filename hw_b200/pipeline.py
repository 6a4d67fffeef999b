"""The whole basecaller path on one B200 at chip size: sensor packets ->
ingest repacking -> the trace-analysis chain with HF metrics (one fused
engine over 4 pools of 4096 lanes, 512-frame chunks, reference defaults;
--streams N: one engine per pool on N streams) ->
BAZ encoding with the preliminary HQ stage (one per pool: production
encoding, 8-chunk metric blocks, the reference's defaults: lookback 10,
preliminary HQ off, so every ZMW is HQ from the first block) ->
every metric block's checkpoint copied to pinned host memory (on a side
stream, overlapping the next steps).

The sensor data are the device trace generator's chunks laid out as the
sensor's packets (blocks of 128 ZMWs x 512 frames), 8 distinct chunks in
device memory used in turn; their generation is outside the timed region.
The run first streams the start-up chunks, then times K steps (CUDA events
on the stream and the host clock around them) and reports ZMW-frames/s for
the whole path, the share of each part, and the checkpoint bytes.

    python -m hw_b200.pipeline [--steps 24] [--warmup-steps 40] [--streams 1]
"""
import argparse
import json
import os
import time

import numpy as np
import torch

from . import abi, filters as Fl, workloads
from .repack import chip_packets

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
POOLS, LANES, F = 4, 4096, 512


def packets_from_traces(tr):
    """[lanes][F][64] traces as the sensor's packet data: blocks of 128 ZMWs
    (two lanes), each [F][128], blocks in ZMW order."""
    lanes = tr.shape[0]
    return tr.view(lanes // 2, 2, F, 64).permute(0, 2, 1, 3).contiguous().view(torch.uint8).reshape(-1)


def run(steps=24, warmup_steps=40, n_inputs=8, pools=POOLS, lanes=LANES, cfg=None, collect=None, streams=1):
    """collect: a list that receives (step, pool, checkpoint copy) for every
    checkpoint (tests).  streams > 1: one fused engine per pool, pool p's
    analysis and BAZ / preliminary HQ stage on stream p mod streams (one
    pool's DME shares the GPU with the other pools' stages); 1: one fused
    engine over every pool on one stream."""
    POOLS, LANES = pools, lanes
    cfg = workloads.chip_config() if cfg is None else cfg
    nz = POOLS * LANES * 64
    gen = Fl.TraceGenerator(POOLS * LANES, workload=1)
    table, nbytes = chip_packets(nz, F)
    packets = []
    for c in range(n_inputs):
        packets.append(packets_from_traces(gen.next(c * F, F)))
        assert packets[-1].numel() == nbytes
    del gen
    rp = Fl.Repacker(nz, LANES, F)
    chunks = rp.new_chunks()
    S = max(1, min(streams, POOLS))
    cart = dict(np.load(os.path.join(ROOT, "hw_b200", "data", "trained_cart.npz")))
    groups = [list(range(POOLS))] if S == 1 else [[p] for p in range(POOLS)]
    units = []
    for g in groups:
        e = Fl.FusedEngine(cfg, [LANES] * len(g), [F] * len(g), pool_ids=g, tuning="auto")
        e.enable_hf_metrics(4096, cfg.frame_rate, True, cart)
        units.append((e, g))
    hq = [Fl.PrelimHq(LANES * 64, chunks_per_block=8, lookback=10, enable=False) for _ in range(POOLS)]
    # each pool's checkpoints land in its own pinned buffer, copied on a side
    # stream that overlaps the next steps' analysis
    host = [torch.empty(min(256 << 20, LANES * 64 * 8 * 64), dtype=torch.uint8, pin_memory=True) for _ in range(POOLS)]
    copy_stream = torch.cuda.Stream()
    copied = [None] * POOLS
    s = torch.cuda.current_stream()
    side = [torch.cuda.Stream() for _ in range(S - 1)]
    ev = {k: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for k in ("repack", "analysis")}
    acc = {k: 0.0 for k in ev}
    ck_bytes, ck_count = 0, 0

    def step(c, timed):
        nonlocal ck_bytes, ck_count
        first = c * F
        if timed:
            ev["repack"][0].record(s)
        # the packets of this chunk's frames, in ZMW order
        tab = table.copy()
        tab["start_frame"] = first
        rp(tab, packets[c % n_inputs], first, chunks)
        if timed:
            ev["repack"][1].record(s)
            ev["analysis"][0].record(s)
        for s_ in side:
            s_.wait_stream(s)
        for u, (eng, g) in enumerate(units):
            su = s if u % S == 0 else side[u % S - 1]
            with torch.cuda.stream(su):
                emitted, _ = eng.process([chunks[p] for p in g])
                m_em = eng.metrics_emitted()
                for i, p in enumerate(g):
                    if not emitted[i]:
                        continue
                    pulses, lens, _ = eng.outputs(i)
                    out = hq[p].process(pulses, lens, cfg.max_calls_per_zmw,
                                        metrics=eng.metrics[i] if m_em[i] else None)
                    if out is not None and collect is not None:
                        collect.append((c, p, {k: (v.clone() if torch.is_tensor(v) else v) for k, v in out.items()}))
                    if out is not None:
                        n = out["bytes"].numel()
                        if copied[p] is not None:
                            copied[p].synchronize()   # the pool's previous checkpoint is out
                        if n > host[p].numel():
                            host[p] = torch.empty(n + n // 4, dtype=torch.uint8, pin_memory=True)
                        ready = torch.cuda.Event()
                        ready.record(su)
                        with torch.cuda.stream(copy_stream):
                            copy_stream.wait_event(ready)
                            host[p][:n].copy_(out["bytes"], non_blocking=True)
                            copied[p] = torch.cuda.Event()
                            copied[p].record(copy_stream)
                        if timed:
                            ck_bytes += n
                            ck_count += 1
        for s_ in side:
            s.wait_stream(s_)
        if timed:
            ev["analysis"][1].record(s)

    for c in range(warmup_steps):
        step(c, False)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0.record(s)
    for c in range(warmup_steps, warmup_steps + steps):
        step(c, True)
        for k, (a, b) in ev.items():
            b.synchronize()
            acc[k] += a.elapsed_time(b)
    e1.record(s)
    e1.synchronize()
    copy_stream.synchronize()
    wall = time.perf_counter() - t0
    ms = e0.elapsed_time(e1)
    zf = nz * F * steps
    for e, _ in units:
        e.finish()
        e.close()
    return {"workload": f"sensor packets -> repacking -> chain with HF metrics ({POOLS} pools x {LANES} lanes, "
                        f"{F}-frame chunks, {len(units)} fused engine(s) on {S} stream(s)) -> BAZ encoding + "
                        f"preliminary HQ (per pool) -> checkpoints to pinned host memory; {steps} steps after "
                        f"{warmup_steps}",
            "zmw_frames_per_s": zf / (ms / 1e3), "zmw_frames_per_s_host_clock": zf / wall,
            "ms_per_step": ms / steps,
            "ms_per_step_by_part": {k: v / steps for k, v in acc.items()},
            "checkpoints": ck_count, "checkpoint_bytes_mean": ck_bytes / max(ck_count, 1)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=24)
    ap.add_argument("--warmup-steps", type=int, default=40)
    ap.add_argument("--streams", type=int, default=1, help="one engine per pool on this many streams (1: one engine)")
    a = ap.parse_args()
    print(json.dumps(run(a.steps, a.warmup_steps, streams=a.streams)))


if __name__ == "__main__":
    main()
