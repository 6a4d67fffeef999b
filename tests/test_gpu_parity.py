"""CUDA path vs. CPU oracle, stage by stage, on identical seeded traces.

Every stage is compared bytewise: the kernels keep the reference Host* order
of floating-point operations, so baseline-subtracted traces, statistics,
histogram counts, detection models (fp16), EM diagnostics, labels and pulse
records are expected to be bit-identical.
"""
import numpy as np
import pytest

from hw_b200 import abi, workloads

import harness
import synth

pytestmark = pytest.mark.gpu


def _eq(name, a, b):
    ab = np.ascontiguousarray(a).view(np.uint8)
    bb = np.ascontiguousarray(b).view(np.uint8)
    assert ab.shape == bb.shape, f"{name}: shape {ab.shape} vs {bb.shape}"
    nd = int((ab != bb).sum())
    assert nd == 0, f"{name}: {nd} of {ab.size} bytes differ"


def _compare_chunk(c, ro, rg, lanes, cap):
    assert sorted(ro) == sorted(rg), f"chunk {c}: stages {sorted(ro)} vs {sorted(rg)}"
    for k in ro:
        if k == "pulses":
            po, lo, oo, bo = ro[k]
            pg, lg, og, bg = rg[k]
            _eq(f"chunk {c} pulse lens", lo, lg)
            _eq(f"chunk {c} pulse overflows", oo, og)
            _eq(f"chunk {c} pulse baseline stats", bo, bg)
            for l in range(lanes):
                for z in range(abi.LANE):
                    n = lo[l, z]
                    _eq(f"chunk {c} pulses lane {l} zmw {z}", po[l, z, :n], pg[l, z, :n])
        elif k == "emit":
            assert ro[k] == rg[k]
        else:
            _eq(f"chunk {c} {k}", ro[k], rg[k])


def _lockstep(cfg, tr, F, pool_id=0):
    lanes = tr.shape[0]
    po = harness.Pipeline(harness.OracleBackend(cfg, lanes, F, pool_id), cfg, pool_id)
    pg = harness.Pipeline(harness.GpuBackend(cfg, lanes, F, pool_id), cfg, pool_id)
    stages = set()
    for c in range(tr.shape[1] // F):
        chunk = np.ascontiguousarray(tr[:, c * F:(c + 1) * F])
        eo = eg = None
        try:
            ro = po.process(chunk, c * F)
        except RuntimeError as e:       # a reference assertion (PBException) on this data
            eo = e
        try:
            rg = pg.process(chunk, c * F)
        except RuntimeError as e:
            eg = e
        assert (eo is None) == (eg is None), f"chunk {c}: oracle error {eo!r}, GPU error {eg!r}"
        if eo is not None:
            # both sides must stop with the same reference status code
            status_o = [n for n in abi.STATUS_NAMES.values() if n in str(eo)]
            status_g = [n for n in abi.STATUS_NAMES.values() if n in str(eg)]
            assert status_o == status_g, f"chunk {c}: {eo!r} vs {eg!r}"
            stages.add("error")
            break
        _compare_chunk(c, ro, rg, lanes, cfg.max_calls_per_zmw)
        stages |= set(ro)
    return stages


def test_small_config_bit_exact():
    cfg = workloads.small_config()
    tr = synth.traces(4, 512 * 8, seed=1)
    stages = _lockstep(cfg, tr, 512)
    assert {"bls", "stats", "init_models", "hist", "models", "diag", "labels", "pulses"} <= stages


def test_small_config_longer_run_reestimates():
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    tr = synth.traces(2, 512 * 16, seed=7, gain_sigma=0.2, empty_fraction=0.15, walk_sigma=0.05)
    _lockstep(cfg, tr, 512)


def test_chip_config_dynamic_bit_exact():
    """Reference defaults (MultiScaleLarge, 9216-frame baseliner start-up, dynamic DME)."""
    cfg = workloads.chip_config()
    tr = synth.traces(2, 512 * 32, seed=3, gain_sigma=0.2, empty_fraction=0.15, walk_sigma=0.05)
    stages = _lockstep(cfg, tr, 512)
    assert "models" in stages and "pulses" in stages


@pytest.mark.parametrize("filt", list(abi.FILTER_TYPES))
def test_every_baseline_filter_bit_exact(filt):
    cfg = workloads.small_config()
    cfg.filter_type = abi.FILTER_TYPES[filt]
    tr = synth.traces(2, 512 * 5, seed=11)
    _lockstep(cfg, tr, 512)


@pytest.mark.parametrize("F", [128, 256])
def test_shorter_chunks_bit_exact(F):
    cfg = workloads.small_config()
    tr = synth.traces(2, F * (4096 // F), seed=5)
    _lockstep(cfg, tr, F)


def test_pulse_overflow_counter():
    """High pulse rate with short pulses overflows the 48-call per-ZMW buffer
    (BatchVectors.h:105-119: the call is dropped and counted)."""
    cfg = workloads.small_config()
    cfg.max_calls_per_zmw = 8
    tr = synth.traces(2, 512 * 8, seed=2, width=3.0, ipd=4.0)
    po = harness.Pipeline(harness.OracleBackend(cfg, 2, 512), cfg)
    pg = harness.Pipeline(harness.GpuBackend(cfg, 2, 512), cfg)
    overflow = 0
    for c in range(8):
        chunk = np.ascontiguousarray(tr[:, c * 512:(c + 1) * 512])
        ro, rg = po.process(chunk, c * 512), pg.process(chunk, c * 512)
        _compare_chunk(c, ro, rg, 2, cfg.max_calls_per_zmw)
        if "pulses" in ro:
            overflow += int(ro["pulses"][2].sum())
    assert overflow > 0


def test_int16_extremes_and_flat_traces():
    """Saturated, negative and constant traces exercise the int16 wrap of the
    reference lane arithmetic and the float->int16 conversion rules."""
    cfg = workloads.small_config()
    rng = np.random.default_rng(9)
    tr = synth.traces(2, 512 * 8, seed=4)
    tr[0, :, :8] = 32767
    tr[0, :, 8:16] = -32768
    tr[0, :, 16:24] = 0
    tr[1, :, :4] = rng.integers(-32768, 32767, size=(tr.shape[1], 4), dtype=np.int16)
    _lockstep(cfg, tr, 512)


def test_native_analyzer_matches_stagewise_pipeline():
    """hw_analyzer (C++ state machine) emits the same pulses as the stage-by-stage pipeline."""
    import torch
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    lanes, F, C = 2, 512, 14
    tr = synth.traces(lanes, F * C, seed=21)
    ref = harness.Pipeline(harness.GpuBackend(cfg, lanes, F, 1), cfg, 1)
    an = Fl.BatchAnalyzer(cfg, 1, lanes, F)
    for c in range(C):
        chunk = np.ascontiguousarray(tr[:, c * F:(c + 1) * F])
        r = ref.process(chunk, c * F)
        pulses, lens, ovf, emitted, estimated = an(torch.from_numpy(chunk).cuda(), c * F)
        lens = lens.cpu().numpy()
        if "pulses" in r and r.get("emit", True):
            assert emitted
            pr, lr, orr, _ = r["pulses"]
            assert np.array_equal(lr, lens.astype(np.uint32))
            pg = Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(lanes, 64, cfg.max_calls_per_zmw)
            for l in range(lanes):
                for z in range(64):
                    assert np.array_equal(pr[l, z, :lr[l, z]].view(np.uint8), pg[l, z, :lens[l, z]].view(np.uint8))
        else:
            assert not emitted and lens.sum() == 0
        assert estimated == ("models" in r)


def _fixed_config():
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.FIXED_ESTIMATIONS
    cfg.static_baseline_mean = 0.0
    cfg.static_baseline_variance = 64.0      # the synthetic baseline sigma is 8 DN
    return cfg


def test_fixed_model_bit_exact():
    """FixedModelBatchAnalyzer schedule: label and pulse every chunk with the
    static model (BatchAnalyzer.cpp:119-207)."""
    cfg = _fixed_config()
    tr = synth.traces(2, 512 * 4, seed=17)
    stages = _lockstep(cfg, tr, 512)
    assert "pulses" in stages and "models" not in stages


def test_native_fixed_analyzer_matches_stagewise_pipeline():
    import torch
    from hw_b200 import filters as Fl
    cfg = _fixed_config()
    lanes, F, C = 2, 512, 4
    tr = synth.traces(lanes, F * C, seed=23)
    ref = harness.Pipeline(harness.GpuBackend(cfg, lanes, F), cfg)
    an = Fl.BatchAnalyzer(cfg, 0, lanes, F)
    for c in range(C):
        chunk = np.ascontiguousarray(tr[:, c * F:(c + 1) * F])
        r = ref.process(chunk, c * F)
        pulses, lens, ovf, emitted, estimated = an(torch.from_numpy(chunk).cuda(), c * F)
        assert emitted and not estimated
        pr, lr, _, _ = r["pulses"]
        lens = lens.cpu().numpy()
        assert np.array_equal(lr, lens.astype(np.uint32))
        pg = Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(lanes, 64, cfg.max_calls_per_zmw)
        for l in range(lanes):
            for z in range(64):
                assert np.array_equal(pr[l, z, :lr[l, z]].view(np.uint8), pg[l, z, :lens[l, z]].view(np.uint8))
    m, _ = an.models()
    assert np.array_equal(Fl.struct_to_numpy(m, abi.LANE_MODEL_DT).view(np.uint8),
                          ref.models.view(np.uint8))


def test_analyzer_rejects_out_of_order_chunks():
    import torch
    from hw_b200 import filters as Fl
    from hw_b200.native import HwError
    cfg = workloads.small_config()
    an = Fl.BatchAnalyzer(cfg, 0, 1, 512)
    chunk = torch.zeros((1, 512, 64), dtype=torch.int16, device="cuda")
    an(chunk, 0)
    with pytest.raises(HwError) as e:
        an(chunk, 1024)
    assert e.value.code == 4


def test_generator_reproducible():
    import torch
    from hw_b200 import filters as Fl
    g1 = Fl.TraceGenerator(4, workload=1)
    g2 = Fl.TraceGenerator(4, workload=1)
    a = [g1.next(c * 512, 512).cpu() for c in range(3)]
    b = [g2.next(c * 512, 512).cpu() for c in range(3)]
    for x, y in zip(a, b):
        assert torch.equal(x, y)
    x = a[0].numpy().astype(np.float64)
    assert 150 < np.median(x) < 250


def test_generated_traces_bit_exact_chip_workload():
    """Device-generated chip-workload traces through both paths (dynamic, 2 pools)."""
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    gen = Fl.TraceGenerator(4, workload=1)
    tr = np.concatenate([gen.next(c * 512, 512).cpu().numpy() for c in range(12)], axis=1)
    _lockstep(cfg, tr[:2], 512, pool_id=0)
    _lockstep(cfg, tr[2:], 512, pool_id=1)


def test_uint8_encoding_equals_its_int16_widening():
    """A uint8 chunk (PacketLayout UINT8) goes through the chain exactly like
    the same values widened to int16 (BatchData.h:160-180)."""
    import torch
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    lanes, F, C = 2, 512, 12
    tr = synth.traces(lanes, F * C, seed=41, baseline=60.0)
    tr8 = np.clip(tr, 0, 255).astype(np.uint8)
    a16 = Fl.BatchAnalyzer(cfg, 0, lanes, F)
    a8 = Fl.BatchAnalyzer(cfg, 0, lanes, F)
    b16 = Fl.Baseliner(cfg, 0, lanes, F)
    b8 = Fl.Baseliner(cfg, 0, lanes, F)
    for c in range(C):
        x8 = torch.from_numpy(np.ascontiguousarray(tr8[:, c * F:(c + 1) * F])).cuda()
        x16 = x8.to(torch.int16)
        o16, s16 = b16(x16, c * F)
        o8, s8 = b8(x8, c * F)
        assert torch.equal(o16, o8) and torch.equal(s16, s8)
        p16, l16, v16, e16, t16 = a16(x16, c * F)
        p8, l8, v8, e8, t8 = a8(x8, c * F)
        assert (e16, t16) == (e8, t8)
        assert torch.equal(l16, l8) and torch.equal(v16, v8)
        if e16:
            q16 = Fl.struct_to_numpy(p16, abi.PULSE_DT).reshape(lanes, 64, cfg.max_calls_per_zmw)
            q8 = Fl.struct_to_numpy(p8, abi.PULSE_DT).reshape(lanes, 64, cfg.max_calls_per_zmw)
            n = l16.cpu().numpy()
            for l in range(lanes):
                for z in range(64):
                    assert np.array_equal(q16[l, z, :n[l, z]].view(np.uint8), q8[l, z, :n[l, z]].view(np.uint8))
    assert e16


def test_pool_set_equals_per_pool_analyzers():
    """hw_pool_set: uneven pools (lane counts 1..5, chunk lengths 128/256/512)
    batched by schedule class (12 pools in 10 classes) give exactly the
    per-pool analyzers' pulses."""
    import torch
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    lanes = [1, 3, 2, 5, 1, 2, 4, 1, 2, 3, 1, 2]
    frames = [512] * 6 + [256] * 3 + [128] * 3
    ps = Fl.PoolSet(cfg, lanes, frames)
    assert ps.launch_groups < len(lanes)
    ans = [Fl.BatchAnalyzer(cfg, p, L, F) for p, (L, F) in enumerate(zip(lanes, frames))]
    gens = [Fl.TraceGenerator(L, workload=2, zmw_offset=1000 * p) for p, L in enumerate(lanes)]
    emitted_any = False
    for step in range(12):
        for p, (g, F) in enumerate(zip(gens, frames)):
            g.next(step * F, F, out=ps.chunk(p))
        em, est = ps.process(step)
        for p, (an, L) in enumerate(zip(ans, lanes)):
            pulses, lens, ovf, e1, s1 = an(ps.chunk(p).clone(), step * frames[p])
            assert (bool(em[p]), bool(est[p])) == (e1, s1)
            if not e1:
                continue
            emitted_any = True
            pp, pl, po = ps.outputs(p)
            assert torch.equal(pl, lens) and torch.equal(po, ovf)
            q0 = Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(L, 64, cfg.max_calls_per_zmw)
            q1 = Fl.struct_to_numpy(pp, abi.PULSE_DT).reshape(L, 64, cfg.max_calls_per_zmw)
            n = lens.cpu().numpy()
            for l in range(L):
                for z in range(64):
                    assert np.array_equal(q0[l, z, :n[l, z]].view(np.uint8), q1[l, z, :n[l, z]].view(np.uint8))
    assert emitted_any


def test_generic_viterbi_rows_bit_exact():
    """Per-analog kinetics break the equal transition constants within the
    9-way rows' source groups: the single-pool labeler's generic rows, stage
    by stage against the oracle."""
    cfg = workloads.small_config()
    for a, (pw, ipd) in enumerate(zip((0.07, 0.08, 0.09, 0.10), (0.12, 0.14, 0.16, 0.18))):
        cfg.analogs[a].pulse_width_s = pw
        cfg.analogs[a].ipd_s = ipd
    tr = synth.traces(4, 512 * 8, seed=3)
    stages = _lockstep(cfg, tr, 512)
    assert {"labels", "pulses"} <= stages
