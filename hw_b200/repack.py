"""Measurement of the ingest repacker (hw_repack_chunk) on the chip
workload: 1,048,576 ZMWs x 512 frames of int16 sensor packets (blocks of 128
ZMWs, 256 blocks and 512 frames per packet, 32 packets, already in device
memory) gathered into 4 pools of 4096 lanes.  Device time with CUDA events
over K calls; the rate is bytes moved (every byte read once and written once)
per second, against the measured HBM copy bandwidth.

    python -m hw_b200.repack [--steps 20] [--zmw 1048576]
"""
import argparse
import json
import os

import numpy as np
import torch

from . import abi, filters as Fl

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def chip_packets(num_zmw=1 << 20, frames=512, block_width=128, blocks=256):
    """Packet table of one chunk (packets in ZMW order, each holding `blocks`
    blocks of `frames` x `block_width` int16 values) and its total bytes."""
    rows, off, z = [], 0, 0
    while z < num_zmw:
        nb = min(blocks, (num_zmw - z) // block_width)
        rows.append((off, z, 0, frames, block_width, nb, 0))
        off += nb * frames * block_width * 2
        z += nb * block_width
    return np.array(rows, abi.SENSOR_PACKET_DT), off


def run(steps=20, warmup=3, num_zmw=1 << 20):
    F, lpp = 512, 4096
    table, nbytes = chip_packets(num_zmw, F)
    data = torch.randint(0, 255, (nbytes,), dtype=torch.uint8, device="cuda")
    rp = Fl.Repacker(num_zmw, lpp, F)
    chunks = rp.new_chunks()
    for _ in range(warmup):
        rp(table, data, 0, chunks)
    torch.cuda.synchronize()
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(steps):
        rp(table, data, 0, chunks)
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            peak = float(json.load(fh)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    gbs = 2 * nbytes / (ms / 1e3) / 1e9
    return {"workload": f"repack {num_zmw} ZMWs x {F} frames int16, {len(table)} packets of 256 x 128-ZMW blocks",
            "bytes_per_call": nbytes, "ms_per_call": ms, "achieved_gbs": gbs, "hbm_peak_gbs": peak,
            "frac_of_measured_hbm": gbs / peak if peak else None,
            "zmw_frames_per_s": num_zmw * F / (ms / 1e3)}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--zmw", type=int, default=1 << 20)
    a = ap.parse_args()
    print(json.dumps(run(a.steps, num_zmw=a.zmw)))


if __name__ == "__main__":
    main()
