"""Analyzer checkpoints (hw_analyzer_state_export / _import): an analyzer
restored from a blob continues exactly like the one that exported it."""
import numpy as np
import pytest

from hw_b200 import abi, workloads

import synth

pytestmark = pytest.mark.gpu


def _run(an, tr, chunks, F):
    import torch
    from hw_b200 import filters as Fl
    out = []
    for c in chunks:
        chunk = torch.from_numpy(np.ascontiguousarray(tr[:, c * F:(c + 1) * F])).cuda()
        pulses, lens, ovf, em, est = an(chunk, c * F)
        out.append((pulses.cpu().numpy().copy(), lens.cpu().numpy().copy(), ovf.cpu().numpy().copy(), em, est))
    m, fi = an.models()
    return out, Fl.struct_to_numpy(m, abi.LANE_MODEL_DT).copy(), fi


@pytest.mark.parametrize("mode", [abi.INITIAL_ESTIMATIONS, abi.DYNAMIC_ESTIMATIONS])
@pytest.mark.parametrize("split", [3, 6, 9])
def test_resume_from_checkpoint_matches_uninterrupted_run(mode, split):
    from hw_b200 import filters as Fl
    cfg = workloads.small_config()
    cfg.model_estimation_mode = mode
    lanes, F, C = 2, 512, 14
    tr = synth.traces(lanes, F * C, seed=31)
    a = Fl.BatchAnalyzer(cfg, 1, lanes, F)
    ref, ref_models, ref_fi = _run(a, tr, range(C), F)
    b = Fl.BatchAnalyzer(cfg, 1, lanes, F)
    _run(b, tr, range(split), F)
    blob = b.export_state()
    c = Fl.BatchAnalyzer(cfg, 1, lanes, F)
    c.import_state(blob)
    got, models, fi = _run(c, tr, range(split, C), F)
    for (p0, l0, o0, e0, s0), (p1, l1, o1, e1, s1) in zip(ref[split:], got):
        assert (e0, s0) == (e1, s1)
        assert np.array_equal(l0, l1) and np.array_equal(o0, o1)
        if e0:
            recs = p0.reshape(lanes, 64, cfg.max_calls_per_zmw, abi.PULSE_DT.itemsize)
            recs1 = p1.reshape(lanes, 64, cfg.max_calls_per_zmw, abi.PULSE_DT.itemsize)
            for l in range(lanes):
                for z in range(64):
                    n = l0[l, z]
                    assert np.array_equal(recs[l, z, :n], recs1[l, z, :n])
    assert np.array_equal(models.view(np.uint8), ref_models.view(np.uint8)) and fi == ref_fi


def test_import_rejects_a_different_analyzer():
    from hw_b200 import filters as Fl
    from hw_b200.native import HwError
    cfg = workloads.small_config()
    a = Fl.BatchAnalyzer(cfg, 0, 2, 512)
    blob = a.export_state()
    with pytest.raises(HwError):
        Fl.BatchAnalyzer(cfg, 0, 3, 512).import_state(blob)
    with pytest.raises(HwError):
        Fl.BatchAnalyzer(cfg, 1, 2, 512).import_state(blob)
    bad = blob.copy()
    bad[:8] = 0
    with pytest.raises(HwError):
        Fl.BatchAnalyzer(cfg, 0, 2, 512).import_state(bad)
