"""Kernel-choice autotuner of the fused engine (hw_fused_set_tuning).

For each chunk length, one engine over a sample of pools is brought to its
steady state (every pool past start-up and in its estimation cycle), then
every candidate kernel choice runs the same number of steps:

  * labeler and pulse accumulator as two kernels, or fused in one kernel
    (labels kept in shared memory instead of a labels batch in HBM);
  * 1, 2 or 4 lanes (64, 128 or 256 threads) a labeler block.

The choices do not change any result (the parity tests run every one), so
they can be switched between steps of one engine.  The score is the device
time of the labeler and pulse stages (stage timers, CUDA events).  Winners
are cached per device name and chunk length in a JSON file that
FusedEngine(tuning="auto") reads.

The tuning key is the chunk length, not the pool size: in the one-launch
engine a block's work depends on its lane's chunk length only, and a pool's
lane count changes nothing but how many blocks the launch has.

    python -m hw_b200.autotune [--frames 128,256,512] [--lanes 16384] [--steps 6]
"""
import argparse
import json
import os

import numpy as np
import torch

from . import abi, filters as Fl, workloads

CANDIDATES = [(fuse, lpc) for fuse in (0, 1) for lpc in (1, 2, 4)]
DEFAULT_FILE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning", "b200.json")


def device_key():
    return torch.cuda.get_device_name(0)


def tune_frames(cfg, F, lanes=16384, pools=8, steps=6):
    """{(fuse, lpc): labeler + pulse ms per step} for chunk length F."""
    lpp = max(lanes // pools, 1)
    eng = Fl.FusedEngine(cfg, [lpp] * pools, [F] * pools)
    gen = Fl.TraceGenerator(lpp * pools, workload=2)
    buf = torch.empty((lpp * pools, F, abi.LANE), dtype=torch.int16, device="cuda")
    step = 0

    def run(n):
        nonlocal step
        for _ in range(n):
            gen.next(step * F, F, out=buf)
            eng.process([buf[p * lpp:(p + 1) * lpp] for p in range(pools)])
            step += 1

    run(workloads.startup_chunks(cfg, pools, F))
    cpe = (max(cfg.min_frames_for_estimate, 1) + F - 1) // F
    n = max(steps, cpe)          # whole estimation cycles: every candidate sees the same DME share
    scores = {}
    for cand in CANDIDATES + CANDIDATES[:1]:       # the first again: warm-up bias check
        eng.set_tuning({F: cand})
        run(1)
        eng.profile(True)
        eng.stage_times()
        run(n)
        t = eng.stage_times()
        eng.profile(False)
        ms = (t["labeler"][0] + t["pulses"][0]) / n
        scores.setdefault(cand, []).append(ms)
    eng.finish()
    eng.close()
    gen.close()
    return {c: float(np.min(v)) for c, v in scores.items()}


def tune(frames=(128, 256, 512), lanes=16384, steps=6, path=DEFAULT_FILE):
    cfg = workloads.chip_config()
    result = {}
    for F in frames:
        sc = tune_frames(cfg, F, lanes=lanes, steps=steps)
        best = min(sc, key=sc.get)
        result[str(F)] = {"fuse_label_pulses": best[0], "labeler_lanes_per_cta": best[1],
                          "ms_per_step": {f"fuse{f}_lpc{l}": v for (f, l), v in sc.items()},
                          "sample": f"{lanes} lanes in 8 pools, chunk length {F}, steady state"}
    data = {}
    if path and os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
    data[device_key()] = result
    if path:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        with open(path, "w") as fh:
            json.dump(data, fh, indent=1, sort_keys=True)
    return result


def load(path=DEFAULT_FILE):
    """{F: (fuse, lanes_per_cta)} cached for this device, or {}."""
    if not os.path.exists(path):
        return {}
    with open(path) as fh:
        data = json.load(fh)
    entry = data.get(device_key(), {})
    return {int(F): (int(v["fuse_label_pulses"]), int(v["labeler_lanes_per_cta"])) for F, v in entry.items()}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--frames", default="128,256,512")
    ap.add_argument("--lanes", type=int, default=16384)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--out", default=DEFAULT_FILE)
    a = ap.parse_args()
    res = tune(tuple(int(x) for x in a.frames.split(",")), a.lanes, a.steps, a.out)
    print(json.dumps(res))


if __name__ == "__main__":
    main()
