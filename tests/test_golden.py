"""The committed golden vectors (tests/golden/small_config_seed1.json, written
by tests/golden/make_golden.py): the oracle must reproduce them on the CPU,
and the CUDA path must reproduce them on the GPU without the oracle running."""
import json
import os

import numpy as np
import pytest

from golden import make_golden as G

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "small_config_seed1.json")


def _load():
    with open(FIXTURE) as f:
        return json.load(f)


def _check(stages, fixture):
    assert len(stages) == len(fixture["stages"])
    for c, (got, want) in enumerate(zip(stages, fixture["stages"])):
        assert sorted(got) == sorted(want), f"chunk {c}: stages {sorted(got)} vs {sorted(want)}"
        for k in want:
            assert got[k] == want[k], f"chunk {c} stage {k} differs from the golden vector"


def test_trace_generator_matches_fixture():
    import synth
    g = _load()
    tr = synth.traces(g["lanes"], g["frames_per_chunk"] * g["chunks"], seed=g["seed"])
    assert G.digest(tr) == g["trace_digest"]


def test_oracle_reproduces_golden_vectors():
    g = _load()
    fresh = G.generate()
    _check(fresh["stages"], g)
    assert fresh["sample"] == g["sample"]


@pytest.mark.gpu
def test_cuda_path_reproduces_golden_vectors():
    import harness
    import synth
    from hw_b200 import abi, workloads
    g = _load()
    cfg = workloads.small_config()
    L, F = g["lanes"], g["frames_per_chunk"]
    tr = synth.traces(L, F * g["chunks"], seed=g["seed"])
    pipe = harness.Pipeline(harness.GpuBackend(cfg, L, F), cfg)
    stages = []
    for c in range(g["chunks"]):
        rec = pipe.process(np.ascontiguousarray(tr[:, c * F:(c + 1) * F]), c * F)
        stages.append(G.stage_digests(rec, cfg.max_calls_per_zmw))
        if c == g["sample"]["models_chunk"]:
            assert rec["models"].view(np.uint16).ravel().tolist() == g["sample"]["models_u16"]
    _check(stages, g)
