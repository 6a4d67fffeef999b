"""Single-ZMW EM fit (hw_dme_em_fit), the engine of the learned initializer.

The fit runs the reference's EM steps per ZMW from the reference start, from
a proposal, or from the better of the two by log-likelihood.  CPU tests check
the oracle's fit for internal consistency; GPU tests check the CUDA fit
bitwise against the oracle in every start mode.
"""
import numpy as np
import pytest

from hw_b200 import workloads

import harness
import synth


class _CaptureBackend(harness.OracleBackend):
    """Records the inputs of the first DME estimate of a pipeline."""

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        self.captured = []

    def estimate(self, hist, stats, hfi, mfi, models):
        self.captured.append((hist.copy(), stats.copy(), hfi, mfi, models.copy()))
        return super().estimate(hist, stats, hfi, mfi, models)


def _dme_inputs(seed=1, lanes=2):
    cfg = workloads.small_config()
    be = _CaptureBackend(cfg, lanes, 512)
    pipe = harness.Pipeline(be, cfg)
    tr = synth.traces(lanes, 512 * 8, seed=seed, gain_sigma=0.2, empty_fraction=0.1)
    for c in range(8):
        pipe.process(np.ascontiguousarray(tr[:, c * 512:(c + 1) * 512]), c * 512)
    assert be.captured
    return cfg, be, be.captured[0]


def test_plain_fit_with_zero_iterations_returns_the_start():
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs()
    p0, it0, ll0 = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=0)
    assert np.isfinite(p0).all()
    assert np.allclose(p0[:, 0:5].sum(1), 1.0, atol=1e-5)          # fractions normalised
    assert (it0[:, 0] == -1).all() and not it0[:, 2].any()
    assert np.array_equal(ll0[:, 0], ll0[:, 1]) and np.array_equal(ll0[:, 1], ll0[:, 2])


def test_proposal_equal_to_plain_start_reproduces_plain_fit():
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs()
    start, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=0)
    pa, ia, la = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=12)
    pb, ib, lb = be.p.em_fit(hist, stats, hfi, mfi, models, mode=1, proposal=start, max_iter=12)
    pc, ic, lc = be.p.em_fit(hist, stats, hfi, mfi, models, mode=2, proposal=start, max_iter=12)
    for p, i, l in ((pb, ib, lb), (pc, ic, lc)):
        assert np.array_equal(pa.view(np.uint32), p.view(np.uint32))
        assert np.array_equal(ia[:, [0, 1, 3]], i[:, [0, 1, 3]])
        assert np.array_equal(la.view(np.uint32), l.view(np.uint32))
    assert not ic[:, 2].any()


def test_bad_proposal_falls_back_to_plain_start():
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs()
    start, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=0)
    bad = start.copy()
    bad[:, 5:10] += 400.0                 # every mode 400 DN too bright
    pa, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=5)
    pb, ib, lb = be.p.em_fit(hist, stats, hfi, mfi, models, mode=2, proposal=bad, max_iter=5)
    assert ib[:, 2].all()
    assert np.array_equal(pa.view(np.uint32), pb.view(np.uint32))
    assert (lb[:, 1] == lb[:, 0]).all()


def test_tolerance_iteration_against_own_fixed_point():
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs()
    ref, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=200)
    _, it, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, target=ref, tol=1e-4, max_iter=200)
    tol_it = it[:, 1]
    assert (tol_it >= 0).all() and (tol_it <= 200).all()
    # from the target itself the distance is 0 at iteration 0
    _, it2, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=1, proposal=ref, target=ref, tol=0.0,
                            max_iter=3)
    assert (it2[:, 1] == 0).all()


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_cuda_fit_matches_oracle(mode):
    import torch
    from hw_b200 import filters as Fl
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs(seed=3)
    lanes = hist.shape[0]
    start, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=0)
    ref, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=60)
    rng = np.random.default_rng(mode)
    prop = (start * (1 + 0.2 * rng.standard_normal(start.shape))).astype(np.float32)
    prop[:, 0:5] = np.abs(prop[:, 0:5]) / np.abs(prop[:, 0:5]).sum(1, keepdims=True)
    prop[:, 10:15] = np.abs(prop[:, 10:15])
    args = dict(target=ref, tol=1e-3, max_iter=25)
    po, io, lo, so = be.p.em_fit(hist, stats, hfi, mfi, models, mode=mode, proposal=None if mode == 0 else prop,
                                 at_stop=True, **args)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    pg, ig, lg, sg = Fl.em_fit(cfg, lanes, Fl.numpy_to_struct(hist), Fl.numpy_to_struct(stats), hfi, mfi,
                               Fl.numpy_to_struct(models), start=mode, proposal=None if mode == 0 else t(prop),
                               target=t(ref), tol=1e-3, max_iter=25, at_stop=True)
    torch.cuda.synchronize()
    assert np.array_equal(po.view(np.uint32), pg.cpu().numpy().view(np.uint32))
    assert np.array_equal(io, ig.cpu().numpy())
    assert np.array_equal(lo.view(np.uint32), lg.cpu().numpy().view(np.uint32))
    sg = sg.cpu().numpy()
    assert np.array_equal(np.isnan(so), np.isnan(sg))
    assert np.array_equal(so[~np.isnan(so)].view(np.uint32), sg[~np.isnan(sg)].view(np.uint32))
    # NaN exactly where no iteration passed the reference's test
    assert np.array_equal(np.isnan(so).all(1), io[:, 0] < 0)


@pytest.mark.gpu
def test_cuda_estimate_from_proposal_matches_oracle():
    """hw_dme_estimate_proposal: the reference estimate (lane-wide stop,
    confidence, blend) from a learned start, bitwise against the oracle."""
    import torch
    from hw_b200 import abi, filters as Fl
    cfg, be, (hist, stats, hfi, mfi, models) = _dme_inputs(seed=6)
    lanes = hist.shape[0]
    start, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=0)
    ref, _, _ = be.p.em_fit(hist, stats, hfi, mfi, models, mode=0, max_iter=80)
    prop = (0.7 * ref + 0.3 * start).astype(np.float32)
    prop[:, 0:5] /= prop[:, 0:5].sum(1, keepdims=True)
    mo, do = be.p.estimate_proposal(hist, stats, hfi, mfi, models, prop)
    dme = Fl.DmeEmEstimator(cfg, 0, lanes)
    m = Fl.numpy_to_struct(models)
    d = dme.estimate_proposal(Fl.numpy_to_struct(hist), hfi, Fl.numpy_to_struct(stats), m, mfi,
                              torch.from_numpy(prop).cuda())
    assert np.array_equal(mo.view(np.uint8), Fl.struct_to_numpy(m, abi.LANE_MODEL_DT).view(np.uint8))
    assert np.array_equal(do.view(np.uint8), Fl.struct_to_numpy(d, abi.DME_DIAG_DT).view(np.uint8))
    # the reference start as proposal reproduces the reference estimate
    mp, dp = be.p.estimate_proposal(hist, stats, hfi, mfi, models, start)
    mr, dr = be.p.estimate(hist, stats, hfi, mfi, models)
    assert np.array_equal(mp.view(np.uint8), mr.view(np.uint8))
