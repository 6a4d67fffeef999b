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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--blocks", type=int, default=12)
    ap.add_argument("--warmup-blocks", type=int, default=11)
    a = ap.parse_args()
    print(json.dumps(run(a.blocks, a.warmup_blocks)))


if __name__ == "__main__":
    main()
