"""Fused chunk engine (hw_chunk_fused): uneven pools in one launch per stage
give exactly the results of one hw_analyzer per pool."""
import os

import numpy as np
import pytest

from hw_b200 import abi, workloads

pytestmark = pytest.mark.gpu

LANES = [1, 3, 2, 5, 1, 2, 4, 1, 2, 3, 1, 2]
FRAMES = [512] * 6 + [256] * 3 + [128] * 3


def _chunks(gens, frames, step, u8):
    import torch
    out = []
    for g, F in zip(gens, frames):
        c = g.next(step * F, F)
        out.append(c.clamp(0, 255).to(torch.uint8) if u8 else c)
    return out


def _same_pulses(cfg, L, a, b, lens):
    from hw_b200 import filters as Fl
    q0 = Fl.struct_to_numpy(a, abi.PULSE_DT).reshape(L, 64, cfg.max_calls_per_zmw)
    q1 = Fl.struct_to_numpy(b, abi.PULSE_DT).reshape(L, 64, cfg.max_calls_per_zmw)
    n = lens.cpu().numpy()
    for l in range(L):
        for z in range(64):
            if not np.array_equal(q0[l, z, :n[l, z]].view(np.uint8), q1[l, z, :n[l, z]].view(np.uint8)):
                return False
    return True


def _compare(mode, graphs, u8, steps, tuning=None, overlap=1):
    import torch
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = mode
    ids = [3 * p + 1 for p in range(len(LANES))]      # stagger classes differ from the positions
    eng = Fl.FusedEngine(cfg, LANES, FRAMES, pool_ids=ids, graphs=graphs, tuning=tuning)
    eng.set_overlap(overlap)
    ans = [Fl.BatchAnalyzer(cfg, i, L, F) for i, L, F in zip(ids, LANES, FRAMES)]
    gens = [Fl.TraceGenerator(L, workload=2, zmw_offset=1000 * p) for p, L in enumerate(LANES)]
    emitted = estimated = 0
    graph_steps = 0
    for step in range(steps):
        chunks = _chunks(gens, FRAMES, step, u8)
        em, est = eng.process(chunks)
        graph_steps += eng.last_step()[1]
        for p, (an, L) in enumerate(zip(ans, LANES)):
            pulses, lens, ovf, e1, s1 = an(chunks[p], step * FRAMES[p])
            assert (bool(em[p]), bool(est[p])) == (e1, s1), (step, p)
            pp, pl, po = eng.outputs(p)
            assert torch.equal(pl, lens) and torch.equal(po, ovf), (step, p)
            if e1:
                emitted += 1
                assert _same_pulses(cfg, L, pulses, pp, lens), (step, p)
            estimated += int(s1)
    eng.finish()
    for p, an in enumerate(ans):
        m0, fi0 = an.models()
        m1, fi1 = eng.models(p)
        assert fi0 == fi1 and torch.equal(m0, m1), p
    return emitted, estimated, graph_steps


@pytest.mark.parametrize("mode", [abi.FIXED_ESTIMATIONS, abi.INITIAL_ESTIMATIONS, abi.DYNAMIC_ESTIMATIONS])
def test_fused_equals_per_pool_analyzers(mode):
    emitted, estimated, _ = _compare(mode, graphs=False, u8=False, steps=28)
    assert emitted > 0
    if mode != abi.FIXED_ESTIMATIONS:
        assert estimated > 0


@pytest.mark.parametrize("overlap", [0, 1, 2])
def test_fused_stream_overlap_modes_equal_per_pool_analyzers(overlap):
    """Every use of the engine's second stream (one stream; the DME beside the
    labeling; the merge, histogram and DME beside it) gives the per-pool
    analyzers' results, with and without graph replay."""
    for graphs in (False, True):
        emitted, estimated, _ = _compare(abi.DYNAMIC_ESTIMATIONS, graphs=graphs, u8=False, steps=28, overlap=overlap)
        assert emitted > 0 and estimated > 0


def test_fused_engines_on_concurrent_streams_equal_per_pool_analyzers():
    """Pool groups, one engine each, run on their own streams at once (the
    layout bench.py times): the engines share no device state, so every
    pool's results equal its per-pool analyzer's, with and without graphs."""
    import torch
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    lanes = [24, 40, 16, 32, 8, 48]
    frames = [512, 512, 256, 512, 128, 256]
    ids = [3 * p + 1 for p in range(len(lanes))]
    groups = [[0, 1], [2, 3], [4], [5]]
    engs = [Fl.FusedEngine(cfg, [lanes[p] for p in g], [frames[p] for p in g], pool_ids=[ids[p] for p in g],
                           graphs=(u % 2 == 1)) for u, g in enumerate(groups)]
    ans = [Fl.BatchAnalyzer(cfg, i, L, F) for i, L, F in zip(ids, lanes, frames)]
    gens = [Fl.TraceGenerator(L, workload=2, zmw_offset=1000 * p) for p, L in enumerate(lanes)]
    main = torch.cuda.current_stream()
    streams = [torch.cuda.Stream() for _ in groups]
    emitted = estimated = 0
    for step in range(28):
        chunks = _chunks(gens, frames, step, False)
        res = []
        for s, e, g in zip(streams, engs, groups):
            s.wait_stream(main)
            with torch.cuda.stream(s):
                res.append(e.process([chunks[p] for p in g]))
        for s in streams:
            main.wait_stream(s)
        for (em, est), e, g in zip(res, engs, groups):
            for i, p in enumerate(g):
                pulses, lens, ovf, e1, s1 = ans[p](chunks[p], step * frames[p])
                assert (bool(em[i]), bool(est[i])) == (e1, s1), (step, p)
                pp, pl, po = e.outputs(i)
                assert torch.equal(pl, lens) and torch.equal(po, ovf), (step, p)
                if e1:
                    emitted += 1
                    assert _same_pulses(cfg, lanes[p], pulses, pp, lens), (step, p)
                estimated += int(s1)
    for e, g in zip(engs, groups):
        e.finish()
        for i, p in enumerate(g):
            m0, fi0 = ans[p].models()
            m1, fi1 = e.models(i)
            assert fi0 == fi1 and torch.equal(m0, m1), p
    assert emitted > 0 and estimated > 0


def test_fused_graphs_replay_identically():
    emitted, estimated, graph_steps = _compare(abi.DYNAMIC_ESTIMATIONS, graphs=True, u8=False, steps=28)
    assert emitted > 0 and estimated > 0
    assert graph_steps > 0


def test_fused_uint8_chunks():
    emitted, _, _ = _compare(abi.DYNAMIC_ESTIMATIONS, graphs=False, u8=True, steps=16)
    assert emitted > 0


def test_fused_rejects_out_of_order_chunks():
    from hw_b200 import filters as Fl
    from hw_b200.native import HwError
    cfg = workloads.small_config()
    eng = Fl.FusedEngine(cfg, [1, 2], [256, 512])
    gens = [Fl.TraceGenerator(L, workload=2) for L in (1, 2)]
    eng.process(_chunks(gens, [256, 512], 0, False))
    eng.next_frame[1] += 512
    with pytest.raises(HwError):
        eng.process(_chunks(gens, [256, 512], 1, False))
    eng.finish()


@pytest.mark.parametrize("tuning", [
    {512: (1, 2), 256: (1, 1), 128: (0, 4)},
    {512: (0, 1), 256: (1, 4), 128: (1, 2)},
    {512: (1, 4), 256: (0, 2), 128: (1, 1)},
])
def test_fused_kernel_variants_equal_per_pool_analyzers(tuning):
    """Every labeler variant (fused with the pulse accumulator or not, 1, 2 or
    4 lanes a block) gives the per-pool analyzers' results."""
    emitted, estimated, _ = _compare(abi.DYNAMIC_ESTIMATIONS, graphs=False, u8=False, steps=28, tuning=tuning)
    assert emitted > 0 and estimated > 0


@pytest.mark.parametrize("mode", [abi.FIXED_ESTIMATIONS, abi.INITIAL_ESTIMATIONS, abi.DYNAMIC_ESTIMATIONS])
def test_fused_hf_metrics_equal_standalone_filter(mode):
    """HF metrics inside hw_chunk_fused equal a standalone hw_hfmetrics filter
    fed by each pool's own analyzer, in the reference's calling pattern."""
    import torch
    from hw_b200 import filters as Fl
    golden = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "hw_b200", "data", "trained_cart.npz")
    cart = dict(np.load(golden))
    cfg = workloads.small_config()
    cfg.model_estimation_mode = mode
    lanes, frames, block = [2, 1, 3], [512, 256, 128], 1024
    eng = Fl.FusedEngine(cfg, lanes, frames)
    eng.enable_hf_metrics(block, cfg.frame_rate, True, cart)
    ans = [Fl.BatchAnalyzer(cfg, p, L, F) for p, (L, F) in enumerate(zip(lanes, frames))]
    hfs = [Fl.HfMetrics(L, block, cfg.frame_rate, True, cart=cart) for L in lanes]
    gens = [Fl.TraceGenerator(L, workload=2, zmw_offset=1000 * p) for p, L in enumerate(lanes)]
    zeros = {L: (torch.zeros((L, 64), dtype=torch.int32, device="cuda"),
                 torch.zeros((L, 64), dtype=torch.float32, device="cuda"),
                 Fl.numpy_to_struct(np.zeros(L, abi.STAT_ACCUM_DT))) for L in set(lanes)}
    blocks = 0
    for step in range(24):
        chunks = _chunks(gens, frames, step, False)
        eng.process(chunks)
        memit = eng.metrics_emitted()
        for p, (an, L, F) in enumerate(zip(ans, lanes, frames)):
            pulses, lens, ovf, em, est = an(chunks[p], step * F)
            runs = mode != abi.DYNAMIC_ESTIMATIONS or em
            if not runs:
                assert memit[p] == 0
                continue
            bs, vit, pd = an.chunk_metrics()
            models, _ = an.models()
            if not em:
                lens_in, vit, pd = zeros[L]
            else:
                lens_in = lens
            got = hfs[p].process(pulses, lens_in, cfg.max_calls_per_zmw, bs, models, vit, pd,
                                 step * F - abi.LATENT_FRAMES, F)
            assert (got is not None) == bool(memit[p]), (step, p)
            if got is not None:
                blocks += 1
                a = Fl.struct_to_numpy(got, abi.BASECALLING_METRICS_DT)
                b = Fl.struct_to_numpy(eng.metrics[p], abi.BASECALLING_METRICS_DT)
                for name in abi.BASECALLING_METRICS_DT.names:
                    assert np.array_equal(a[name], b[name], equal_nan=a[name].dtype.kind == "f"), (step, p, name)
    eng.finish()
    assert blocks > 0


def test_fused_last_diag_equals_per_pool_analyzers():
    """hw_fused_last_diag gives each pool's diagnostics of its latest
    estimate, equal to its per-pool analyzer's; none before the first."""
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    lanes, frames, ids = [3, 2], [512, 256], [1, 4]
    eng = Fl.FusedEngine(cfg, lanes, frames, pool_ids=ids)
    ans = [Fl.BatchAnalyzer(cfg, i, n, F) for i, n, F in zip(ids, lanes, frames)]
    gens = [Fl.TraceGenerator(n, workload=2, zmw_offset=1000 * p) for p, n in enumerate(lanes)]
    assert eng.last_diag(0) is None
    seen = 0
    for step in range(24):
        chunks = [g.next(step * F, F) for g, F in zip(gens, frames)]
        eng.process(chunks)
        for p, an in enumerate(ans):
            an(chunks[p], step * frames[p])
            d0, d1 = an.last_diag(), eng.last_diag(p)
            assert (d0 is None) == (d1 is None), (step, p)
            if d0 is not None:
                seen += 1
                assert np.array_equal(Fl.struct_to_numpy(d0, abi.DME_DIAG_DT).view(np.uint8),
                                      Fl.struct_to_numpy(d1, abi.DME_DIAG_DT).view(np.uint8)), (step, p)
    eng.finish()
    assert seen > 0
