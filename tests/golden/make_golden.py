"""Writes tests/golden/small_config_seed1.json: per chunk, the SHA-256 of
every stage output of the oracle on the small configuration (2 lanes = 128
ZMWs, 8 chunks of 512 frames, tests/synth.py traces with seed 1), plus the
first pulses of four ZMWs and the estimated models in full.

These are regression vectors of this repository's oracle (the reference
itself cannot be built here); the oracle's agreement with the reference is
pinned separately by tests/test_oracle_kat.py.

    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

LANES, F, CHUNKS, SEED = 2, 512, 8, 1
OUT = os.path.join(HERE, "small_config_seed1.json")


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).view(np.uint8).tobytes()).hexdigest()


def stage_digests(rec, cap):
    out = {}
    for k, v in sorted(rec.items()):
        if k == "emit":
            out[k] = bool(v)
        elif k == "pulses":
            p, lens, ovf, bls = v
            # only the written records count: later slots are unspecified
            valid = np.concatenate([p[l, z, :lens[l, z]].view(np.uint8).ravel()
                                    for l in range(p.shape[0]) for z in range(p.shape[1])])
            out["pulses"] = digest(valid)
            out["pulse_lens"] = digest(lens)
            out["pulse_overflows"] = digest(ovf)
            out["pulse_baseline_stats"] = digest(bls)
        else:
            out[k] = digest(v)
    return out


def generate():
    import harness
    import synth
    from hw_b200 import abi, workloads
    cfg = workloads.small_config()
    tr = synth.traces(LANES, F * CHUNKS, seed=SEED)
    pipe = harness.Pipeline(harness.OracleBackend(cfg, LANES, F), cfg)
    chunks, sample = [], {}
    for c in range(CHUNKS):
        rec = pipe.process(np.ascontiguousarray(tr[:, c * F:(c + 1) * F]), c * F)
        chunks.append(stage_digests(rec, cfg.max_calls_per_zmw))
        if "models" in rec:
            m = rec["models"]
            sample["models_chunk"] = c
            sample["models_u16"] = m.view(np.uint16).ravel().tolist()
        if "pulses" in rec and "pulses_chunk" not in sample:
            p, lens, _, _ = rec["pulses"]
            sample["pulses_chunk"] = c
            sample["pulses"] = {f"{l}/{z}": [[int(x["start"]), int(x["width"]), int(x["mean_signal"]),
                                              int(x["mid_signal"]), int(x["max_signal"]), float(x["signal_m2"]),
                                              int(x["label"]), int(x["is_reject"])]
                                             for x in p[l, z, :lens[l, z]]]
                                for l, z in ((0, 0), (0, 17), (1, 5), (1, 63))}
    return {"lanes": LANES, "frames_per_chunk": F, "chunks": CHUNKS, "seed": SEED,
            "config": "small_config", "trace_digest": digest(tr), "stages": chunks, "sample": sample}


if __name__ == "__main__":
    g = generate()
    with open(OUT, "w") as f:
        json.dump(g, f, indent=1)
    print("wrote", OUT)
