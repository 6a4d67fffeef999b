"""Failures injected on the host -- inverted histogram bounds, a frame gap --
come back as C-ABI status codes, without a device fault, and the handle
keeps working afterwards."""
import numpy as np
import pytest

from hw_b200 import abi, workloads

HW_ERR_FRAME_ORDER, HW_ERR_NUMERIC = 4, 9


@pytest.mark.gpu
def test_histogram_reports_inverted_bounds_and_recovers():
    """Bounds the reference refuses (UHistogramSimd.cpp:66-96: the lower
    bound must be below the upper one): the reset kernel's check sets the
    deferred error word, the call returns HW_ERR_NUMERIC, and a valid reset
    then works."""
    import torch
    from hw_b200 import filters as Fl
    from hw_b200.native import HwError
    cfg = workloads.small_config()
    lanes = 2
    h = Fl.TraceHistogramAccumulator(cfg, 0, lanes)
    b = np.zeros(lanes, abi.HIST_BOUNDS_DT)
    b["lower_bounds"] = 200.0
    b["upper_bounds"] = 100.0
    d_b = torch.from_numpy(b.view(np.uint8).reshape(-1).copy()).cuda()
    with pytest.raises(HwError) as e:
        h.reset_from_bounds(d_b)
    assert e.value.code == HW_ERR_NUMERIC
    b["lower_bounds"] = -20.0
    d_b = torch.from_numpy(b.view(np.uint8).reshape(-1).copy()).cuda()
    h.reset_from_bounds(d_b)
    out, _ = h.histogram()
    hist = Fl.struct_to_numpy(out, abi.LANE_HIST_DT)
    assert np.allclose(hist["low_bound"], -20.0)


@pytest.mark.gpu
def test_fused_engine_rejects_a_frame_gap_and_continues():
    """A chunk whose first frame skips ahead is refused (HW_ERR_FRAME_ORDER,
    nothing launched); the right chunk is then taken as if nothing happened:
    the results equal an engine that never saw the bad call."""
    import torch
    from hw_b200 import filters as Fl
    from hw_b200.native import HwError
    cfg = workloads.small_config()
    lanes, F = 2, 512
    gen = Fl.TraceGenerator(2 * lanes, workload=1)
    chunks = [gen.next(c * F, F).clone() for c in range(12)]
    a = Fl.FusedEngine(cfg, [lanes, lanes], [F, F])
    b = Fl.FusedEngine(cfg, [lanes, lanes], [F, F])
    for c, ch in enumerate(chunks):
        parts = [ch[:lanes].contiguous(), ch[lanes:].contiguous()]
        if c == 5:
            a.next_frame[1] += F
            with pytest.raises(HwError) as e:
                a.process(parts)
            assert e.value.code == HW_ERR_FRAME_ORDER
            a.next_frame[1] -= F
        ea, _ = a.process(parts)
        eb, _ = b.process(parts)
        assert (ea == eb).all()
        for p in range(2):
            pa, la, _ = a.outputs(p)
            pb, lb, _ = b.outputs(p)
            assert torch.equal(la, lb)
            if ea[p]:
                # the valid records (slots past a ZMW's count are unspecified)
                ra = Fl.struct_to_numpy(pa, abi.PULSE_DT).reshape(lanes * 64, -1)
                rb = Fl.struct_to_numpy(pb, abi.PULSE_DT).reshape(lanes * 64, -1)
                n = la.cpu().numpy().reshape(-1)
                for z in range(lanes * 64):
                    assert ra[z, :n[z]].tobytes() == rb[z, :n[z]].tobytes()
