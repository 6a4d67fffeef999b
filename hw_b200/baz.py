"""Measurement of BAZ pulse encoding (hw_baz_encode) on chip-sized chunks:
the pulses of one 512-frame chunk of 1,048,576 ZMWs (4 pools of 4096 lanes;
the chain's own pulses of one pool, analysed from synthetic traces and
repeated over the four pools), 48 pulse slots a ZMW, already in device
memory.  Device time with CUDA events over K calls (each call is the sizing
pass, the offset scan and the encoding pass, and one stream synchronisation).
The rate is the algorithmic bytes -- the pulses read twice (sizing and
encoding), the pulse counts, the offsets and the encoded bytes written -- per
second, against the measured HBM copy bandwidth; pulses/s beside it.

    python -m hw_b200.baz [--steps 20] [--preset production|internal]
"""
import argparse
import json
import os

import numpy as np
import torch

from . import abi, filters as Fl, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PULSE_BYTES = abi.PULSE_DT.itemsize


def chain_pulses(lanes=4096, frames=512, chunks=10):
    """The pulses and counts of the last of `chunks` chunks the chain analysed
    (short start-up configuration, synthetic traces)."""
    cfg = workloads.small_config()
    gen = Fl.TraceGenerator(lanes, workload=1, zmw_offset=0)
    an = Fl.BatchAnalyzer(cfg, 0, lanes, frames)
    out = None
    for c in range(chunks):
        pulses, lens, ovf, em, est = an(gen.next(c * frames, frames), c * frames)
        if em:
            out = (pulses.clone(), lens.clone())
    assert out is not None, "the chain emitted no pulses"
    return out[0], out[1], cfg.max_calls_per_zmw


def run(steps=20, warmup=3, preset="production", pools=4):
    which = abi.BAZ_PRODUCTION if preset == "production" else abi.BAZ_INTERNAL
    pulses, lens, cap = chain_pulses()
    pulses = pulses.repeat(pools)
    lens = lens.reshape(-1).repeat(pools).contiguous()
    nz = lens.numel()
    enc = Fl.BazEncoder(nz, preset=which)
    for _ in range(warmup):
        data, off = enc(pulses, lens, cap)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        data, off = enc(pulses, lens, cap)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    n_pulses = int(lens.to(torch.int64).sum().item())
    out_bytes = data.numel()
    algo = 2 * n_pulses * PULSE_BYTES + 2 * nz * 4 + out_bytes + 3 * (nz + 1) * 8
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = float(json.load(fh)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    gbs = algo / (ms / 1e3) / 1e9
    return {"workload": f"BAZ {preset} encoding of one 512-frame chunk of {nz} ZMWs, {cap} pulse slots a ZMW",
            "pulses_per_call": n_pulses, "encoded_bytes": out_bytes, "algorithmic_bytes": algo,
            "ms_per_call": ms, "achieved_gbs": gbs, "hbm_peak_gbs": peak,
            "frac_of_measured_hbm": gbs / peak if peak else None, "pulses_per_s": n_pulses / (ms / 1e3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--preset", default="production", choices=["production", "internal"])
    a = ap.parse_args()
    print(json.dumps(run(a.steps, preset=a.preset)))


if __name__ == "__main__":
    main()
