"""Trace-histogram binning at its edges, CUDA against the oracle bit for bit:
values exactly on the first and last bin edge, one bin outside either end,
the int16 extremes, and bin sizes so small that (x - lower) / binSize passes
2^31, where the reference's floor-and-cast (TraceHistogramAccumHost.cpp:140-169
through UHistogramSimd::AddDatum) yields INT_MIN and the frame counts as a low
outlier.  Chunks of 512 and 256 frames take the kernel's split path (the
chunk's halves binned as two chains), 40 frames the single-chain path; the
edge-classifier state and the counts carry across the calls."""
import numpy as np
import pytest

from hw_b200 import abi, workloads

LANE = abi.LANE


def _bounds(lanes):
    b = np.zeros(lanes, abi.HIST_BOUNDS_DT)
    for l in range(lanes):
        for z in range(LANE):
            g = (l * LANE + z) % 4
            if g == 0:      # bin size exactly 1: integer x sits on bin edges
                lo, hi = -100.0, 200.0
            elif g == 1:    # bin size 1e-7: x >= 215 gives a quotient above 2^31
                lo, hi = 0.0, 3e-5
            elif g == 2:    # half-integer offsets
                lo, hi = -0.5, 299.5
            else:
                lo = float(-50 - 7 * z)
                hi = lo + 40.0 + 3.0 * l
            b[l]["lower_bounds"][z] = lo
            b[l]["upper_bounds"][z] = hi
    return b


def _traces(rng, lanes, frames):
    """Runs of 3 to 9 equal frames (so the edge classifier passes most
    frames) drawn from values at and around the bin edges."""
    vals = np.array([-32768, -102, -101, -100, -99, -1, 0, 1, 5, 19, 20, 21, 99, 100, 101,
                     198, 199, 200, 201, 214, 215, 216, 299, 300, 5000, 32767], np.int16)
    out = np.empty((lanes, frames, LANE), np.int16)
    for l in range(lanes):
        for z in range(LANE):
            f = 0
            while f < frames:
                n = int(rng.integers(3, 10))
                out[l, f:f + n, z] = vals[rng.integers(len(vals))]
                f += n
    return out


def _models(lanes):
    m = np.zeros(lanes, abi.LANE_MODEL_DT)
    m["baseline"]["means"][:] = abi.f32_to_f16(0.0)
    m["baseline"]["vars"][:] = abi.f32_to_f16(100.0)     # edge threshold 20
    return m


@pytest.mark.gpu
def test_histogram_edges_bit_exact():
    import torch
    from hw_b200 import filters as Fl
    import oracle
    cfg = workloads.small_config()
    lanes = 3
    rng = np.random.default_rng(2024)
    bounds, models = _bounds(lanes), _models(lanes)
    ref = oracle.Pool(cfg, lanes, 512, 0)
    ref.hist_reset_from_bounds(bounds)
    gpu = Fl.TraceHistogramAccumulator(cfg, 0, lanes)
    gpu.reset_from_bounds(torch.from_numpy(bounds.view(np.uint8).reshape(-1).copy()).cuda())
    d_models = torch.from_numpy(models.view(np.uint8).reshape(-1).copy()).cuda()
    first = 0
    for frames in (512, 40, 256, 40, 512):
        tr = _traces(rng, lanes, frames)
        fi = (first, first + frames)
        ref.hist_add(tr, fi, models)
        gpu.add_batch(torch.from_numpy(tr).cuda(), fi, d_models)
        first += frames
        want, wfi = ref.hist_get()
        out, gfi = gpu.histogram()
        got = Fl.struct_to_numpy(out, abi.LANE_HIST_DT)
        assert gfi == wfi
        for k in ("bin_count", "outlier_count_low", "outlier_count_high", "low_bound", "bin_size"):
            assert np.array_equal(got[k].view(np.uint8), want[k].view(np.uint8)), (frames, k)
    # the quotient-above-2^31 class was reached: those ZMWs counted low outliers
    low = want["outlier_count_low"].reshape(-1)
    assert low[1::4].sum() > 0 and want["outlier_count_high"].reshape(-1)[0::4].sum() > 0
