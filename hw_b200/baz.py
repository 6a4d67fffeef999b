"""Measurement of BAZ pulse encoding (hw_baz_encode_async) on chip-sized
chunks: the pulses of consecutive 512-frame chunks of 1,048,576 ZMWs (4
pools of 4096 lanes; the chain's own pulses of one pool, analysed from
synthetic traces and repeated over the four pools), 48 pulse slots a ZMW,
every chunk already in device memory (1 GB each).  Device time with CUDA events over K encodings enqueued back to back
(one launch each); the synchronous call (hw_baz_encode, which waits for the
total) is timed beside it.  The rate is the algorithmic bytes -- the pulses
read once, the pulse counts, the delta state read and written, the offsets
and the encoded bytes written -- per second, against the measured HBM copy
bandwidth; pulses/s beside it.

    python -m hw_b200.baz [--steps 20] [--warmup 3] [--preset production|internal] [--pools 4]
"""
import argparse
import json
import os

import numpy as np
import torch

from . import abi, filters as Fl, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PULSE_BYTES = abi.PULSE_DT.itemsize


def chain_pulses(n_chunks, lanes=4096, frames=512):
    """The pulses and counts of `n_chunks` consecutive chunks the chain emitted
    (short start-up configuration, synthetic traces)."""
    cfg = workloads.small_config()
    gen = Fl.TraceGenerator(lanes, workload=1, zmw_offset=0)
    an = Fl.BatchAnalyzer(cfg, 0, lanes, frames)
    out, c = [], 0
    while len(out) < n_chunks:
        pulses, lens, ovf, em, est = an(gen.next(c * frames, frames), c * frames)
        if em:
            out.append((pulses.clone(), lens.clone()))
        c += 1
    return out, cfg.max_calls_per_zmw


def run(steps=20, warmup=3, preset="production", pools=4):
    which = abi.BAZ_PRODUCTION if preset == "production" else abi.BAZ_INTERNAL
    pool_chunks, cap = chain_pulses(warmup + steps)
    # every chunk on all pools: one encoder over pools x 262,144 ZMWs
    chunks = [(p.repeat(pools), l.reshape(-1).repeat(pools).contiguous()) for p, l in pool_chunks]
    del pool_chunks
    nz = chunks[0][1].numel()
    n_pulses = sum(int(l.to(torch.int64).sum().item()) for _, l in chunks[warmup:]) / steps
    enc = Fl.BazEncoder(nz, preset=which)
    first, _ = enc(*chunks[0], cap)
    out = torch.empty(2 * first.numel() + (16 << 20), dtype=torch.uint8, device="cuda")
    offsets = torch.empty(nz + 1, dtype=torch.int64, device="cuda")
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        for c in range(warmup):
            fn(c)
        torch.cuda.synchronize()
        e0.record(s)
        for c in range(warmup, warmup + steps):
            fn(c)
        e1.record(s)
        e1.synchronize()
        return e0.elapsed_time(e1) / steps

    # a fresh encoder for each loop, so both see the chunks in order
    enc = Fl.BazEncoder(nz, preset=which)
    sizes = []

    def enqueue(c):
        enc.enqueue(*chunks[c], cap, out, offsets)
    ms = timed(enqueue)
    out_bytes = enc.result()                     # the last chunk's bytes
    sync = Fl.BazEncoder(nz, preset=which)

    def call(c):
        data, _ = sync(*chunks[c], cap)
        sizes.append(data.numel())
    ms_sync = timed(call)
    assert sizes[-1] == out_bytes
    out_bytes = sum(sizes[warmup:]) / steps
    algo = n_pulses * PULSE_BYTES + nz * 4 + 2 * nz * 8 + (nz + 1) * 8 + out_bytes
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = float(json.load(fh)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    gbs = algo / (ms / 1e3) / 1e9
    return {"workload": f"BAZ {preset} encoding of {steps} consecutive 512-frame chunks of {nz} ZMWs "
                        f"({cap} pulse slots a ZMW), each chunk resident in device memory",
            "pulses_per_call": n_pulses, "encoded_bytes_per_call": out_bytes, "algorithmic_bytes": algo,
            "ms_per_call": ms, "ms_per_sync_call": ms_sync, "achieved_gbs": gbs, "hbm_peak_gbs": peak,
            "frac_of_measured_hbm": gbs / peak if peak else None, "pulses_per_s": n_pulses / (ms / 1e3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--preset", default="production", choices=["production", "internal"])
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--pools", type=int, default=4)
    a = ap.parse_args()
    print(json.dumps(run(a.steps, a.warmup, preset=a.preset, pools=a.pools)))


if __name__ == "__main__":
    main()
