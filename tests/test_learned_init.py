"""Learned DME initializer: the CPU reference network against finite
differences, the CUDA features / targets / proposals / forward pass /
gradients against the CPU reference, and a small training run that must beat
the plain EM start."""
import numpy as np
import pytest

import mlp_ref as R

from test_em_fit import _dme_inputs


def _random_net(rng, scale=1.0):
    p = np.zeros(R.N_PARAMS, np.float32)
    p[R.OFF_W1:R.OFF_B1] = rng.standard_normal(R.OFF_B1 - R.OFF_W1) * np.sqrt(2.0 / R.FEAT) * scale
    p[R.OFF_B1:R.OFF_W2] = 0.1 * rng.standard_normal(R.HID)
    p[R.OFF_W2:R.OFF_B2] = rng.standard_normal(R.HID * R.HID) * np.sqrt(2.0 / R.HID) * scale
    p[R.OFF_B2:R.OFF_W3] = 0.1 * rng.standard_normal(R.HID)
    w3 = np.zeros((R.OUT, R.HID), np.float32)
    w3[:R.OUT_USED] = rng.standard_normal((R.OUT_USED, R.HID)) * np.sqrt(2.0 / R.HID)
    p[R.OFF_W3:R.OFF_B3] = w3.ravel()
    p[R.OFF_B3:R.OFF_B3 + R.OUT_USED] = 0.1 * rng.standard_normal(R.OUT_USED)
    norm = np.zeros(2 * R.FEAT + 2 * R.OUT, np.float32)
    norm[R.FEAT:2 * R.FEAT] = 1.0
    norm[2 * R.FEAT + R.OUT:] = 1.0
    return p, norm


def test_reference_gradients_match_finite_differences():
    """The CPU reference's backward pass is the derivative of its forward
    pass (float64 network, no bf16 rounding)."""
    rng = np.random.default_rng(0)
    p, norm = _random_net(rng)
    feat = rng.standard_normal((6, R.FEAT)).astype(np.float32)
    tgt = rng.standard_normal((6, R.OUT)).astype(np.float32)
    p64 = p.astype(np.float64)
    _, g = R.loss_and_gradients(p64, norm, feat, tgt, bf16_round=False)
    for idx in list(rng.choice(R.N_PARAMS, 40, replace=False)) + [R.OFF_B3, R.OFF_B1 + 3, R.OFF_W3 + 5]:
        h = 1e-5
        pp, pm = p64.copy(), p64.copy()
        pp[idx] += h
        pm[idx] -= h
        lp, _ = R.loss_and_gradients(pp, norm, feat, tgt, bf16_round=False)
        lm, _ = R.loss_and_gradients(pm, norm, feat, tgt, bf16_round=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-4 * abs(fd), (idx, fd, g[idx])


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.gpu
def test_features_targets_and_proposal_kernels_match_reference():
    import torch
    from hw_b200 import filters as Fl, learned_init as L
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs(seed=4)
    lanes = hist.shape[0]
    pool = L.Pool(cfg, lanes, Fl.numpy_to_struct(hist), Fl.numpy_to_struct(stats), hfi, Fl.numpy_to_struct(models),
                  mfi)
    f = L.features(pool).cpu().numpy()
    assert np.allclose(f, R.features(hist, stats), rtol=1e-6, atol=1e-7)
    params, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=30)
    t = L.targets(pool, _dev(params)).cpu().numpy()
    assert np.allclose(t, R.targets(params, hist, cfg.shot_var_coeff), rtol=1e-5, atol=1e-5)
    net = L.Network(max_batch=256, seed=3)
    _, norm = net.get()
    rng = np.random.default_rng(2)
    norm[2 * R.FEAT:2 * R.FEAT + R.OUT_USED] = rng.standard_normal(R.OUT_USED)
    norm[2 * R.FEAT + R.OUT:2 * R.FEAT + R.OUT + R.OUT_USED] = rng.uniform(0.5, 2.0, R.OUT_USED)
    net.set(norm=norm)
    y = rng.standard_normal((lanes * 64, R.OUT)).astype(np.float32)
    P = net.proposal(pool, _dev(y)).cpu().numpy()
    torch.cuda.synchronize()
    assert np.allclose(P, R.proposal(y, norm, hist), rtol=1e-5, atol=1e-5)


@pytest.mark.gpu
def test_fused_proposal_equals_the_three_steps():
    """hw_learned_init_propose (features, tensor-core forward pass and EM
    start in one launch) gives the bits of features -> forward -> proposal,
    on an odd lane count (a half-filled last tile) and a random network."""
    from hw_b200 import filters as Fl, learned_init as L
    cfg, _, (hist, stats, hfi, mfi, models) = _dme_inputs(seed=6, lanes=3)
    lanes = hist.shape[0]
    pool = L.Pool(cfg, lanes, Fl.numpy_to_struct(hist), Fl.numpy_to_struct(stats), hfi, Fl.numpy_to_struct(models),
                  mfi)
    rng = np.random.default_rng(9)
    p, norm = _random_net(rng, scale=0.7)
    norm[:R.FEAT] = 0.05 * rng.standard_normal(R.FEAT)
    norm[R.FEAT:2 * R.FEAT] = rng.uniform(0.5, 2.0, R.FEAT)
    norm[2 * R.FEAT:2 * R.FEAT + R.OUT_USED] = rng.standard_normal(R.OUT_USED)
    norm[2 * R.FEAT + R.OUT:2 * R.FEAT + R.OUT + R.OUT_USED] = rng.uniform(0.5, 2.0, R.OUT_USED)
    net = L.Network(max_batch=256, seed=3)
    net.set(p, norm)
    three = net.proposal(pool, net.forward(L.features(pool))).cpu().numpy()
    fused = net.propose(pool).cpu().numpy()
    net.forward_status()
    assert np.isfinite(three).all()
    assert three.tobytes() == fused.tobytes()


@pytest.mark.gpu
def test_forward_and_gradients_match_reference():
    """BF16 tensor-core forward and backward against the CPU reference with
    the same BF16 rounding points; they differ only by FP32 accumulation order
    (and the occasional activation that rounds to the neighbouring BF16)."""
    from hw_b200 import learned_init as L
    rng = np.random.default_rng(5)
    net = L.Network(max_batch=512, seed=11)
    p, norm = _random_net(rng)
    norm[:R.FEAT] = 0.1 * rng.standard_normal(R.FEAT)
    norm[R.FEAT:2 * R.FEAT] = rng.uniform(0.5, 2.0, R.FEAT)
    norm[2 * R.FEAT + R.OUT:2 * R.FEAT + R.OUT + R.OUT_USED] = rng.uniform(0.5, 2.0, R.OUT_USED)
    net.set(p, norm)
    n = 300
    feat = rng.standard_normal((n, R.FEAT)).astype(np.float32)
    tgt = rng.standard_normal((n, R.OUT)).astype(np.float32)
    y = net.forward(_dev(feat)).cpu().numpy()
    net.forward_status()
    y_ref, _ = R.forward(p, norm, feat)
    err = np.abs(y - y_ref)
    assert err.max() <= 2e-2 * np.abs(y_ref).max() and np.median(err) <= 2e-3 * np.abs(y_ref).mean()
    loss, g = net.gradients(_dev(feat), _dev(tgt))
    loss_ref, g_ref = R.loss_and_gradients(p, norm, feat, tgt)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    g = g.cpu().numpy()
    for name, a, b in (("W1", R.OFF_W1, R.OFF_B1), ("b1", R.OFF_B1, R.OFF_W2), ("W2", R.OFF_W2, R.OFF_B2),
                       ("b2", R.OFF_B2, R.OFF_W3), ("W3", R.OFF_W3, R.OFF_B3), ("b3", R.OFF_B3, R.N_PARAMS)):
        ga, gb = g[a:b].astype(np.float64), g_ref[a:b]
        rel = np.linalg.norm(ga - gb) / max(np.linalg.norm(gb), 1e-30)
        assert rel <= 1e-2, (name, rel)
    # parameters and normalisation survive a round trip through the handle
    p2, n2 = net.get()
    assert np.array_equal(p2, p) and np.array_equal(n2, norm)


@pytest.mark.gpu
def test_training_beats_plain_start():
    """A small training run (2 pools x 512 lanes of the uneven-pool
    generator) gives, on a held-out pool, an EM start that meets the
    reference's stopping rule in at most half the iterations of the
    reference start, meets the parameter-step rule no later, and reaches the
    plain EM's fixed point no more than 5% later; the proposal is taken (not
    the fallback) for most ZMWs."""
    from hw_b200 import learned_init as L
    net, m = L.run(train_pools=2, eval_pools=1, lanes=512, fit_iters=400, epochs=25, batch=1024, seed=3)
    assert m["resolved_fraction"] > 0.5
    assert 2 * m["reference_criterion_iters_learned_mean"] <= m["reference_criterion_iters_plain_mean"], m
    assert m["step_criterion_iters_learned_mean"] <= m["step_criterion_iters_plain_mean"], m
    assert m["em_iters_learned_mean"] <= 1.05 * m["em_iters_plain_mean"], m
    assert m["fallback_rate"] < 0.5, m


@pytest.mark.gpu
def test_analyzer_with_learned_start_runs_dynamic_schedule():
    """hw_analyzer_set_learned_init: a dynamic-estimation analyzer starts its
    estimates from the network's proposal and still emits pulses and finite
    models; detaching the network restores the reference start."""
    import torch
    from hw_b200 import abi, filters as Fl, learned_init as L, workloads
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    net, _ = L.run(train_pools=1, eval_pools=1, lanes=256, fit_iters=200, epochs=5, batch=1024, seed=2)
    lanes, F = 64, 512
    gen = Fl.TraceGenerator(lanes, workload=1)
    an = Fl.BatchAnalyzer(cfg, 0, lanes, F)
    an.set_learned_init(net)
    estimated = emitted = 0
    for c in range(16):
        _, lens, _, em, est = an(gen.next(c * F, F), c * F)
        estimated += int(est)
        emitted += int(em)
    assert estimated >= 2 and emitted > 0 and int(lens.sum()) > 0
    m, _ = an.models()
    means = abi.f16_to_f32(Fl.struct_to_numpy(m, abi.LANE_MODEL_DT)["analogs"]["means"])
    assert np.isfinite(means).all()
    an.set_learned_init(None)
    an(gen.next(16 * F, F), 16 * F)
    torch.cuda.synchronize()


@pytest.mark.gpu
def test_analyzers_on_streams_with_learned_start_equal_serial():
    """Analyzers with the learned start run at once on two streams, each
    stream with its own copy of the network (a network handle holds its
    forward pass's scratch), give the results of the same analyzers run one
    after another on one stream."""
    import torch
    from hw_b200 import abi, filters as Fl, learned_init as L, workloads
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    net, _ = L.run(train_pools=1, eval_pools=1, lanes=256, fit_iters=200, epochs=5, batch=1024, seed=2)
    net2 = L.Network(max_batch=net.max_batch)
    net2.set(*net.get())
    lanes, F, pools = 32, 512, 4
    serial = [Fl.BatchAnalyzer(cfg, p, lanes, F) for p in range(pools)]
    conc = [Fl.BatchAnalyzer(cfg, p, lanes, F) for p in range(pools)]
    for p in range(pools):
        serial[p].set_learned_init(net)
        conc[p].set_learned_init(net if p % 2 == 0 else net2)
    gens = [Fl.TraceGenerator(lanes, workload=2, zmw_offset=5000 * p) for p in range(pools)]
    main = torch.cuda.current_stream()
    side = [torch.cuda.Stream(), torch.cuda.Stream()]
    estimated = emitted = 0
    for c in range(20):
        chunks = [g.next(c * F, F) for g in gens]
        for s in side:
            s.wait_stream(main)
        res = []
        for p in range(pools):
            with torch.cuda.stream(side[p % 2]):
                res.append(conc[p](chunks[p], c * F))
        for s in side:
            main.wait_stream(s)
        for p in range(pools):
            pulses0, lens0, ovf0, em0, est0 = serial[p](chunks[p], c * F)
            pulses1, lens1, ovf1, em1, est1 = res[p]
            assert (em0, est0) == (em1, est1), (c, p)
            assert torch.equal(lens0, lens1) and torch.equal(ovf0, ovf1), (c, p)
            q0 = Fl.struct_to_numpy(pulses0, abi.PULSE_DT).reshape(lanes * 64, cfg.max_calls_per_zmw)
            q1 = Fl.struct_to_numpy(pulses1, abi.PULSE_DT).reshape(lanes * 64, cfg.max_calls_per_zmw)
            n = np.minimum(lens0.cpu().numpy().reshape(-1), cfg.max_calls_per_zmw)
            for z in range(lanes * 64):
                assert np.array_equal(q0[z, :n[z]].view(np.uint8), q1[z, :n[z]].view(np.uint8)), (c, p, z)
            estimated += int(est0)
            emitted += int(em0)
    for p in range(pools):
        m0, fi0 = serial[p].models()
        m1, fi1 = conc[p].models()
        assert fi0 == fi1 and torch.equal(m0, m1), p
    assert estimated >= pools and emitted > 0
    net2.close()


@pytest.mark.gpu
@pytest.mark.parametrize("graphs", [False, True])
def test_fused_engine_with_learned_start_equals_analyzers(graphs):
    """hw_fused_set_learned_init: pools of uneven sizes and chunk lengths in
    one engine, every estimate from the network's proposal, give the results
    of one analyzer per pool with the same network (graphs replay the plans of
    the steps, which include the estimating pools); the models differ from
    those of the reference start."""
    import torch
    from hw_b200 import abi, filters as Fl, learned_init as L, workloads
    cfg = workloads.small_config()
    cfg.model_estimation_mode = abi.DYNAMIC_ESTIMATIONS
    net, _ = L.run(train_pools=1, eval_pools=1, lanes=256, fit_iters=200, epochs=5, batch=1024, seed=2)
    lanes, frames, ids = [24, 40, 16], [512, 256, 512], [1, 4, 7]
    eng = Fl.FusedEngine(cfg, lanes, frames, pool_ids=ids, graphs=graphs)
    eng.set_learned_init(net)
    plain = Fl.FusedEngine(cfg, lanes, frames, pool_ids=ids)
    ans = [Fl.BatchAnalyzer(cfg, i, n, F) for i, n, F in zip(ids, lanes, frames)]
    for a in ans:
        a.set_learned_init(net)
    gens = [Fl.TraceGenerator(n, workload=2, zmw_offset=1000 * p) for p, n in enumerate(lanes)]
    estimated = emitted = 0
    for step in range(28):
        chunks = [g.next(step * F, F) for g, F in zip(gens, frames)]
        em, est = eng.process(chunks)
        plain.process(chunks)
        for p, (an, n) in enumerate(zip(ans, lanes)):
            pulses, lens, ovf, e1, s1 = an(chunks[p], step * frames[p])
            assert (bool(em[p]), bool(est[p])) == (e1, s1), (step, p)
            pp, pl, po = eng.outputs(p)
            assert torch.equal(pl, lens) and torch.equal(po, ovf), (step, p)
            if e1:
                emitted += 1
                q0 = Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(n * 64, cfg.max_calls_per_zmw)
                q1 = Fl.struct_to_numpy(pp, abi.PULSE_DT).reshape(n * 64, cfg.max_calls_per_zmw)
                cnt = np.minimum(lens.cpu().numpy().reshape(-1), cfg.max_calls_per_zmw)
                for z in range(n * 64):
                    assert np.array_equal(q0[z, :cnt[z]].view(np.uint8), q1[z, :cnt[z]].view(np.uint8)), (step, p, z)
            estimated += int(s1)
    eng.finish()
    plain.finish()
    differs = False
    for p, an in enumerate(ans):
        m0, fi0 = an.models()
        m1, fi1 = eng.models(p)
        assert fi0 == fi1 and torch.equal(m0, m1), p
        m2, _ = plain.models(p)
        differs |= not torch.equal(m1, m2)
    assert estimated >= 3 and emitted > 0 and differs
