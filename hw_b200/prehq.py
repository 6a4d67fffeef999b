"""Measurement of the preliminary HQ stage (hw_prelim_hq_process) at chip size:
1,048,576 ZMWs, 512-frame chunks, 8 chunks a metric block, a lookback of 10
blocks, the placeholder HQ rule on (throttle 0.10), production encoding.
Input: the chain's own pulses of 24 consecutive chunks of a 4096-lane pool
(on all four pools), resident, used in turn.  Device time with CUDA events
over K chunks after W warm-up chunks (every call synchronises once, a block's
end twice more); reported per chunk, and per metric-block checkpoint with its
bytes copied.

    python -m hw_b200.prehq [--blocks 12] [--warmup-blocks 11]
"""
import argparse
import json
import os

import torch

from . import abi, filters as Fl
from .baz import chain_pulses

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run(blocks=12, warmup_blocks=11, pools=4, chunks_per_block=8, lookback=10, n_inputs=24):
    pool_chunks, cap = chain_pulses(n_inputs)
    chunks = [(p.repeat(pools), l.reshape(-1).repeat(pools).contiguous()) for p, l in pool_chunks]
    del pool_chunks
    nz = chunks[0][1].numel()
    st = Fl.PrelimHq(nz, chunks_per_block=chunks_per_block, lookback=lookback, enable=True, throttle=0.10)
    s = torch.cuda.current_stream()
    c = 0
    for _ in range(warmup_blocks * chunks_per_block):   # fills the window; HQ marking starts at block 10
        st.process(*chunks[c % n_inputs], cap)
        c += 1
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ck_bytes, ck_hq = [], []
    e0.record(s)
    for _ in range(blocks * chunks_per_block):
        out = st.process(*chunks[c % n_inputs], cap)
        c += 1
        if out is not None:
            ck_bytes.append(out["bytes"].numel())
            ck_hq.append(out["num_hq"])
    e1.record(s)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    n_chunks = blocks * chunks_per_block
    # the chunk encoding alone, for the checkpoint's share
    enc = Fl.BazEncoder(nz)
    e0.record(s)
    for k in range(n_chunks):
        enc(*chunks[k % n_inputs], cap)
    e1.record(s)
    e1.synchronize()
    ms_enc = e0.elapsed_time(e1)
    per_block_ck = (ms - ms_enc) / blocks
    mean_ck = sum(ck_bytes) / len(ck_bytes)
    return {"workload": f"preliminary HQ stage, {nz} ZMWs, 512-frame chunks, {chunks_per_block} chunks a metric block, "
                        f"lookback {lookback} blocks, placeholder HQ rule (throttle 0.10), production encoding; "
                        f"{blocks} blocks timed after {warmup_blocks}",
            "ms_per_chunk": ms / n_chunks, "ms_per_chunk_encoding_only": ms_enc / n_chunks,
            "ms_per_checkpoint": per_block_ck, "checkpoint_bytes_mean": mean_ck,
            "checkpoint_gbs": 2 * mean_ck / (per_block_ck / 1e3) / 1e9 if per_block_ck > 0 else None,
            "num_hq_after": ck_hq[-1], "zmw_frames_per_s": nz * 512 * n_chunks / (ms / 1e3)}


def _hf_blocks(lanes, n, seed=1):
    """n blocks of synthetic HF metrics (hw_basecalling_metrics lanes) whose
    activity labels change in about a third of the ZMWs from block to block."""
    import numpy as np
    rng = np.random.default_rng(seed)
    L, A = (lanes, abi.LANE), (lanes, abi.NUM_ANALOGS, abi.LANE)
    out = []
    lab = rng.integers(0, 4, L)
    for _ in range(n):
        m = np.zeros(lanes, abi.BASECALLING_METRICS_DT)
        lab = np.where(rng.random(L) < 0.35, rng.integers(0, 4, L), lab)
        m["activity_label"] = lab
        for f in ("num_pulse_frames", "num_base_frames", "num_bases", "num_pulses", "num_sandwiches"):
            m[f] = rng.integers(0, 3000, L)
        m["num_frames"], m["num_frames_baseline"] = 4096, rng.integers(0, 3000, L)
        m["frame_baseline_dws"] = rng.normal(0, 6, L)
        m["frame_baseline_variance_dws"] = rng.uniform(10, 90, L)
        m["num_pk_mid_frames"] = rng.integers(0, 400, A)
        m["pk_mid_signal"] = rng.uniform(0, 400, A) * m["num_pk_mid_frames"]
        m["pk_max"], m["pk_zvar"], m["bp_zvar"] = rng.uniform(0, 900, A), rng.uniform(0, 9, A), rng.uniform(0, 2, A)
        out.append(torch.from_numpy(m.view(np.uint8)).cuda())
    return out


def run_metric_side(blocks=12, warmup_blocks=11, lanes=16384, chunks_per_block=8, lookback=10, enable=True):
    """The metric side (hw_prelim_hq_metrics) at chip size: two stages on the
    same empty pulse chunks and HF metrics, with and without the metric side;
    the difference per metric block is its cost (the add at the block's
    last chunk, sizing, scan, placement and writing of the blocks)."""
    nz = lanes * abi.LANE
    hf = _hf_blocks(lanes, 4)
    cap = 4
    pulses = torch.zeros(nz * cap * abi.PULSE_DT.itemsize, dtype=torch.uint8, device="cuda")
    lens = torch.zeros(nz, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream()
    res = {}
    for metrics in (False, True):
        st = Fl.PrelimHq(nz, chunks_per_block=chunks_per_block, lookback=lookback, enable=enable, throttle=0.10,
                         metrics=metrics)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        blocks_out = []
        for b in range(warmup_blocks + blocks):
            if b == warmup_blocks:
                torch.cuda.synchronize()
                e0.record(s)
            for c in range(chunks_per_block):
                st.process(pulses, lens, cap, metrics=hf[b % len(hf)] if c == chunks_per_block - 1 else None)
            if metrics and b >= warmup_blocks:
                blocks_out.append(st.metric_checkpoint()["total"])
        e1.record(s)
        e1.synchronize()
        res["with" if metrics else "without"] = e0.elapsed_time(e1) / blocks
        if metrics:
            res["metric_blocks_per_checkpoint"] = sum(blocks_out) / len(blocks_out)
        st.close()
    per_block = res["with"] - res["without"]
    return {"workload": f"metric side of the preliminary HQ stage, {nz} ZMWs, {chunks_per_block} chunks a metric block, "
                        f"lookback {lookback}, preliminary HQ {'on' if enable else 'off'} (throttle 0.10), "
                        f"synthetic HF metrics; {blocks} blocks timed after {warmup_blocks}",
            "ms_per_block_with": res["with"], "ms_per_block_without": res["without"],
            "metric_side_ms_per_block": per_block,
            "metric_blocks_per_checkpoint": res["metric_blocks_per_checkpoint"]}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--blocks", type=int, default=12)
    ap.add_argument("--warmup-blocks", type=int, default=11)
    ap.add_argument("--metric-side", action="store_true", help="time the metric side instead")
    a = ap.parse_args()
    if a.metric_side:
        print(json.dumps({"production": run_metric_side(a.blocks, a.warmup_blocks, enable=True),
                          "complete": run_metric_side(a.blocks, a.warmup_blocks, enable=False)}))
    else:
        print(json.dumps(run(a.blocks, a.warmup_blocks)))


if __name__ == "__main__":
    main()
