"""hw_dme_estimate_noalloc: the DME estimate for callers that cannot allocate.

Code that runs where cudaMalloc is off limits (inside a custom allocator's
callbacks, or a real-time pipeline whose device memory is fixed up front)
cannot create an hw_dme handle, because the handle allocates its EM scratch.
hw_dme_estimate_noalloc runs the same kernel with the scratch in a fixed
file-scope device array instead, so it allocates nothing.  This test checks
that it returns exactly what hw_dme_estimate returns, on two different
inputs in a row (the second call reuses the array the first one filled).
"""
import ctypes as C

import numpy as np
import pytest

from hw_b200 import abi, workloads

import harness
import synth

pytestmark = pytest.mark.gpu


class _CaptureBackend(harness.GpuBackend):
    """Records the inputs of every DME estimate the pipeline runs."""

    def __init__(self, *a, **kw):
        super().__init__(*a, **kw)
        self.captured = []

    def estimate(self, hist, stats, hfi, mfi, models):
        self.captured.append((hist.copy(), stats.copy(), hfi, mfi, models.copy()))
        return super().estimate(hist, stats, hfi, mfi, models)


def _estimate_inputs(seed, lanes=4, chunks=8):
    cfg = workloads.small_config()
    be = _CaptureBackend(cfg, lanes, 512)
    pipe = harness.Pipeline(be, cfg)
    tr = synth.traces(lanes, 512 * chunks, seed=seed)
    for c in range(chunks):
        pipe.process(np.ascontiguousarray(tr[:, c * 512:(c + 1) * 512]), c * 512)
    assert be.captured, "the schedule ran no estimate"
    return cfg, be.captured[0]


def _run_noalloc(cfg, lanes, hist, stats, hfi, mfi, models):
    import torch
    from hw_b200 import filters as Fl
    from hw_b200.native import check, lib
    # keep every device buffer referenced until the call has completed
    h = Fl.numpy_to_struct(hist)
    s = Fl.numpy_to_struct(stats)
    m = Fl.numpy_to_struct(models)
    d = Fl.struct_buffer(abi.DME_DIAG_DT, lanes)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib().hw_dme_estimate_noalloc(C.byref(cfg), lanes, C.c_void_p(h.data_ptr()), C.c_void_p(s.data_ptr()),
                                        abi.FrameInterval(*hfi), abi.FrameInterval(*mfi), C.c_void_p(m.data_ptr()),
                                        C.c_void_p(d.data_ptr()), stream))
    return Fl.struct_to_numpy(m, abi.LANE_MODEL_DT), Fl.struct_to_numpy(d, abi.DME_DIAG_DT)


def _run_handle(cfg, lanes, hist, stats, hfi, mfi, models):
    from hw_b200 import filters as Fl
    dme = Fl.DmeEmEstimator(cfg, 0, lanes)
    m = Fl.numpy_to_struct(models)
    d = dme.estimate(Fl.numpy_to_struct(hist), hfi, Fl.numpy_to_struct(stats), m, mfi)
    return Fl.struct_to_numpy(m, abi.LANE_MODEL_DT), Fl.struct_to_numpy(d, abi.DME_DIAG_DT)


def test_noalloc_estimate_matches_handle_estimate_on_two_calls():
    for seed in (1, 2):
        cfg, (hist, stats, hfi, mfi, models) = _estimate_inputs(seed)
        lanes = hist.shape[0]
        m_ref, d_ref = _run_handle(cfg, lanes, hist, stats, hfi, mfi, models)
        m_na, d_na = _run_noalloc(cfg, lanes, hist, stats, hfi, mfi, models)
        assert np.array_equal(m_ref.view(np.uint8), m_na.view(np.uint8)), f"models differ (seed {seed})"
        assert np.array_equal(d_ref.view(np.uint8), d_na.view(np.uint8)), f"diagnostics differ (seed {seed})"


def test_noalloc_rejects_more_than_128_lanes():
    from hw_b200.native import lib
    cfg = workloads.small_config()
    z = C.c_void_p(1)
    rc = lib().hw_dme_estimate_noalloc(C.byref(cfg), 129, z, z, abi.FrameInterval(0, 512), abi.FrameInterval(0, 512),
                                       z, None, None)
    assert rc == 1
    assert b"128" in lib().hw_last_error_string()
