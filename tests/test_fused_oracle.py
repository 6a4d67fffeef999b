"""The uneven-pool engine (hw_chunk_fused) against the
oracle directly: every pool of one fused engine, fed the uneven-pool
generator's traces (per-ZMW amplitude factors, pulse rates up to 0.12 a
frame, so 512-frame chunks overflow the 48 pulse slots and the overflow
counter of DT/BatchVectors.h:105-119 counts the dropped pulses), must give,
step by step, exactly what one oracle analyzer per pool gives: the same
emit / estimate decisions, pulse counts, overflow counts and pulse records
byte for byte, and at the end the same detection models.

Pools mix lane counts {1, 2, 37, 64} with chunk lengths {128, 256, 512};
pool ids differ from the positions so the stagger classes differ.  Both the
reference defaults (MultiScaleLarge, dynamic estimation every 4000 frames)
and the shortened small configuration (TwoScaleMedium, single estimate) run.
"""
import numpy as np
import pytest

from hw_b200 import abi, workloads

pytestmark = pytest.mark.gpu

POOLS = [(1, 128), (2, 256), (37, 512), (64, 128), (2, 512), (37, 256)]   # (lanes, frames per chunk)
IDS = [5, 2, 11, 0, 7, 3]


def _run(cfg, steps):
    import torch
    from hw_b200 import filters as Fl
    import harness
    lanes = [L for L, _ in POOLS]
    frames = [F for _, F in POOLS]
    eng = Fl.FusedEngine(cfg, lanes, frames, pool_ids=IDS)
    pipes = [harness.Pipeline(harness.OracleBackend(cfg, L, F, pid), cfg, pid) for (L, F), pid in zip(POOLS, IDS)]
    gens = [Fl.TraceGenerator(L, workload=2, zmw_offset=4096 * p) for p, L in enumerate(lanes)]
    cap = cfg.max_calls_per_zmw
    emitted = overflowed = estimated = 0
    for step in range(steps):
        chunks = [g.next(step * F, F) for g, F in zip(gens, frames)]
        em, est = eng.process(chunks)
        torch.cuda.synchronize()
        for p, ((L, F), pipe) in enumerate(zip(POOLS, pipes)):
            rec = pipe.process(chunks[p].cpu().numpy(), step * F)
            o_est = "models" in rec
            o_emit = "pulses" in rec and rec.get("emit", True)
            assert bool(est[p]) == o_est, (step, p, "estimate")
            assert bool(em[p]) == o_emit, (step, p, "emit")
            estimated += int(o_est)
            if not o_emit:
                continue
            emitted += 1
            want_p, want_len, want_ovf, _ = rec["pulses"]
            pp, pl, po = eng.outputs(p)
            got_len = pl.cpu().numpy().astype(np.uint32).reshape(L, 64)
            got_ovf = po.cpu().numpy().astype(np.uint32).reshape(L, 64)
            assert np.array_equal(got_len, want_len), (step, p, "lens")
            assert np.array_equal(got_ovf, want_ovf), (step, p, "overflows")
            overflowed += int((want_ovf > 0).sum())
            got_p = Fl.struct_to_numpy(pp, abi.PULSE_DT).reshape(L, 64, cap)
            for l in range(L):
                for z in range(64):
                    n = min(int(want_len[l, z]), cap)
                    assert np.array_equal(got_p[l, z, :n].view(np.uint8), want_p[l, z, :n].view(np.uint8)), \
                        (step, p, l, z)
    eng.finish()
    for p, pipe in enumerate(pipes):
        m, _ = eng.models(p)
        got = Fl.struct_to_numpy(m, abi.LANE_MODEL_DT)
        assert np.array_equal(got.view(np.uint8), pipe.models.view(np.uint8)), p
    return emitted, estimated, overflowed


def test_uneven_pools_reference_defaults_equal_oracle():
    cfg = workloads.chip_config()
    # 128-frame pools need 9216 frames of baseliner start-up, the stagger,
    # 1000 frames of statistics and an estimation period before they emit
    emitted, estimated, overflowed = _run(cfg, steps=140)
    assert emitted > 0 and estimated > 0 and overflowed > 0, (emitted, estimated, overflowed)


def test_uneven_pools_small_configuration_equal_oracle():
    cfg = workloads.small_config()
    emitted, estimated, overflowed = _run(cfg, steps=40)
    assert emitted > 0 and estimated > 0 and overflowed > 0, (emitted, estimated, overflowed)


def _varied_kinetics(cfg):
    """Per-analog pulse widths and inter-pulse distances: the 9-way rows'
    transition constants then differ within each source group, so the
    labeler takes its generic rows instead of the grouped ones."""
    for a, (pw, ipd) in enumerate(zip((0.07, 0.08, 0.09, 0.10), (0.12, 0.14, 0.16, 0.18))):
        cfg.analogs[a].pulse_width_s = pw
        cfg.analogs[a].ipd_s = ipd
    return cfg


def _grouped(cfg):
    import oracle
    T = oracle.transition_matrix(cfg)
    rows = T[[0, 5, 6, 7, 8]]
    return bool((rows[:, 5:9] == rows[:, 5:6]).all() and (rows[:, 9:13] == rows[:, 9:10]).all())


def test_uneven_pools_generic_viterbi_rows_equal_oracle():
    cfg = _varied_kinetics(workloads.small_config())
    assert _grouped(workloads.small_config()) and not _grouped(cfg)
    emitted, estimated, overflowed = _run(cfg, steps=40)
    assert emitted > 0 and estimated > 0, (emitted, estimated, overflowed)
