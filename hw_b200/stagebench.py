"""Small-case runner of the full chain, for profiling one stage at a time.

    python -m hw_b200.stagebench --lanes 2048 --chunks 10 [--config small|chip]

Runs the native analyzer over device-generated traces (workload 1 generator)
and prints the per-stage device time of the last chunks.  With the small
configuration labeling starts at chunk 7, so `--chunks 10` gives three
labeler launches; 2048 lanes make a 134 MB chunk (larger than the 126 MB L2).
"""
import argparse
import json

import torch

from . import abi, filters as Fl, workloads


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--lanes", type=int, default=2048)
    ap.add_argument("--chunks", type=int, default=10)
    ap.add_argument("--frames", type=int, default=512)
    ap.add_argument("--config", choices=["small", "chip"], default="small")
    a = ap.parse_args()
    cfg = workloads.small_config() if a.config == "small" else workloads.chip_config()
    an = Fl.BatchAnalyzer(cfg, 0, a.lanes, a.frames)
    gen = Fl.TraceGenerator(a.lanes, workload=1)
    buf = torch.empty((a.lanes, a.frames, 64), dtype=torch.int16, device="cuda")
    an.profile(True)
    emitted = 0
    for c in range(a.chunks):
        gen.next(c * a.frames, a.frames, out=buf)
        _, lens, _, em, _ = an(buf, c * a.frames)
        if em and not emitted:
            # the first chunk that runs every stage loads their kernels (lazy
            # module loading): its times are left out
            torch.cuda.synchronize()
            an.stage_times()
        emitted += int(em)
    torch.cuda.synchronize()
    times = an.stage_times()
    out = {"lanes": a.lanes, "chunks": a.chunks, "emitted_chunks": emitted,
           "pulses_last_chunk": int(lens.sum().item()),
           "stage_ms_total": {k: v[0] for k, v in times.items()},
           "stage_launches": {k: v[1] for k, v in times.items()}}
    diag = an.last_diag()
    if diag is not None:
        d = Fl.struct_to_numpy(diag, abi.DME_DIAG_DT)
        it = d["lane_iterations"].astype(float)
        out["dme_lane_iterations"] = {"mean": float(it.mean()), "max": int(it.max()),
                                      "hist": [int((d["lane_iterations"] == i).sum()) for i in range(21)]}
        out["dme_converged_fraction"] = float(d["converged"].mean())
    print(json.dumps(out))


if __name__ == "__main__":
    main()
