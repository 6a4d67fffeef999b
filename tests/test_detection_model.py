"""Detection-model conversion and confidence decay, pinned by the reference's
own unit tests (src/basecaller/basecaller/test/TestDetectionModelHost.cpp).

LaneDetectionModelConversion (:54-116): a DetectionModelHost built from the
mock lane model (LaneDetectionModel.h:187-212: baseline weight 0.40, mean 0,
variance 1; analogs weight 0.15, means 4/6/9/13, variances 1.1-1.4) is
changed one property at a time; each change is visible against a copy, and
after ExportTo + re-import the copy agrees again to half precision
(|a - b| < 0.000978 max(a, b)).  EvolveConfidence (:118-128): confidence 1
halves over one half-life between interval centres, then decays by
sqrt(0.5) over half a half-life.

Both are run on the oracle (CPU) and on the library's own conversion kernels
(the functions the DME uses), which must also equal the oracle bit for bit
on random values, including variances above the fp16 clamp of 65000, NaN,
infinities and subnormal halves.
"""
import ctypes as C

import numpy as np
import pytest

from hw_b200 import abi

HALF_EPS = np.float32(0.000978)


def _h(x):
    return np.float16(x).view(np.uint16)


def mock_lane_model(lanes=1):
    m = np.zeros(lanes, abi.LANE_MODEL_DT)
    m["baseline"]["weights"] = _h(0.40)
    m["baseline"]["means"] = _h(0.0)
    m["baseline"]["vars"] = _h(1.0)
    for i, (mu, var) in enumerate(zip((4.0, 6.0, 9.0, 13.0), (1.1, 1.2, 1.3, 1.4))):
        m["analogs"][:, i]["weights"] = _h(0.15)
        m["analogs"][:, i]["means"] = _h(mu)
        m["analogs"][:, i]["vars"] = _h(var)
    m["confidence"] = _h(0.0)
    return m


def equal_to_half_precision(a, b):
    return bool(np.all(np.abs(a - b) < HALF_EPS * np.maximum(a, b)))


class OracleModels:
    def __init__(self):
        import oracle
        self.o = oracle

    def imp(self, models):
        return self.o.detection_model_import(models)

    def exp(self, params):
        return self.o.detection_model_export(params)

    def evolve(self, params, fi_from, fi_to, half_life):
        return self.o.detection_model_evolve_confidence(params, fi_from, fi_to, half_life)


class GpuModels:
    def __init__(self):
        import torch
        from hw_b200 import native
        self.torch = torch
        self.lib = native.lib()
        self.check = native.check

    def _dev(self, a):
        t = self.torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).copy()).cuda()
        return t, C.c_void_p(t.data_ptr())

    def imp(self, models):
        m, pm = self._dev(models)
        out = self.torch.zeros(len(models) * 16 * abi.LANE, dtype=self.torch.float32, device="cuda")
        self.check(self.lib.hw_detection_model_import(pm, len(models), C.c_void_p(out.data_ptr()), None))
        self.torch.cuda.synchronize()
        return out.cpu().numpy().reshape(len(models), 16, abi.LANE)

    def exp(self, params):
        p, pp = self._dev(np.ascontiguousarray(params, np.float32))
        out = self.torch.zeros(len(params) * abi.LANE_MODEL_DT.itemsize, dtype=self.torch.uint8, device="cuda")
        self.check(self.lib.hw_detection_model_export(pp, len(params), C.c_void_p(out.data_ptr()), None))
        self.torch.cuda.synchronize()
        return out.cpu().numpy().view(abi.LANE_MODEL_DT)

    def evolve(self, params, fi_from, fi_to, half_life):
        p, pp = self._dev(np.ascontiguousarray(params, np.float32))
        self.check(self.lib.hw_detection_model_evolve_confidence(
            pp, len(params), abi.FrameInterval(*fi_from), abi.FrameInterval(*fi_to), C.c_float(half_life), None))
        self.torch.cuda.synchronize()
        return p.cpu().numpy().view(np.float32).reshape(params.shape)


# rows of the float parameters: baseline weight/mean/var, analog i at 3+3i..5+3i, confidence 15
def _check_conversion(B):
    dmh0 = B.imp(mock_lane_model())
    dmh1 = dmh0.copy()
    assert np.array_equal(dmh0, dmh1)
    state = {"dmh1": dmh1}

    def round_trip():
        ldm = B.exp(dmh0)
        state["dmh1"] = B.imp(ldm)

    def change(row, delta):
        dmh0[:, row] += np.float32(delta)
        assert not equal_to_half_precision(dmh0[:, row], state["dmh1"][:, row]), row
        round_trip()
        assert equal_to_half_precision(dmh0[:, row], state["dmh1"][:, row]), row

    change(0, 0.02)     # baseline weight
    change(1, 1.0)      # baseline mean
    change(2, 2.0)      # baseline variance
    for i in range(4):
        change(3 + 3 * i, 0.01)
        change(4 + 3 * i, 1.0)
        change(5 + 3 * i, 2.0)
    change(15, 0.2)     # confidence


def _check_evolve(B):
    p = B.imp(mock_lane_model())
    p[:, 15] = 1.0
    p = B.evolve(p, (0, 100), (100, 200), 100.0)
    assert np.all(p[:, 15] == np.float32(0.5))
    p = B.evolve(p, (100, 200), (200, 300), 200.0)
    expect = np.float32(0.5) * np.sqrt(np.float32(0.5))
    assert np.all(np.abs(p[:, 15] - expect) < np.float32(1e-6) * expect)


def test_oracle_lane_model_conversion():
    _check_conversion(OracleModels())


def test_oracle_evolve_confidence():
    _check_evolve(OracleModels())


def test_oracle_export_clamps_variances():
    O = OracleModels()
    p = O.imp(mock_lane_model())
    p[:, 2] = 1e6
    p[:, 5] = 70000.0
    m = O.exp(p)
    assert np.all(m["baseline"]["vars"] == _h(65000.0))      # half(65000) = 64992
    assert np.all(m["analogs"][:, 0]["vars"] == _h(65000.0))


def _random_params(rng, lanes):
    p = rng.normal(0, 1, (lanes, 16, abi.LANE)).astype(np.float32) * np.float32(50.0)
    p[:, [2, 5, 8, 11, 14]] = np.abs(p[:, [2, 5, 8, 11, 14]]) * np.float32(2000.0)   # variances past 65000 too
    p[0, 1, :8] = [np.nan, np.inf, -np.inf, 1e-7, -1e-7, 6e-8, 70000.0, -70000.0]
    p[0, 2, :4] = [np.nan, np.inf, 65000.0, 64991.0]
    return p


@pytest.mark.gpu
def test_gpu_lane_model_conversion():
    _check_conversion(GpuModels())


@pytest.mark.gpu
def test_gpu_evolve_confidence():
    _check_evolve(GpuModels())


@pytest.mark.gpu
def test_gpu_conversion_equals_oracle_on_random_values():
    G, O = GpuModels(), OracleModels()
    rng = np.random.default_rng(7)
    p = _random_params(rng, 3)
    _same_bits(G.exp(p).view(np.uint16).view(np.float16), O.exp(p).view(np.uint16).view(np.float16))
    bits = rng.integers(0, 1 << 16, 3 * abi.LANE_MODEL_DT.itemsize // 2, dtype=np.uint16)
    models = bits.view(abi.LANE_MODEL_DT)
    _same_bits(G.imp(models), O.imp(models))
    p[:, 15] = np.abs(p[:, 15])
    for fi0, fi1, hl in (((0, 512), (4096, 8192), 4096.0), ((100, 200), (0, 50), 12000.0), ((5, 6), (5, 7), 3.5)):
        _same_bits(G.evolve(p, fi0, fi1, hl), O.evolve(p, fi0, fi1, hl))


def _same_bits(a, b):
    """Bit-equal, except that a NaN only has to meet a NaN (NaN payloads of
    conversions are not part of the reference's contract)."""
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb)
    ui = np.uint16 if a.dtype == np.float16 else np.uint32
    assert np.array_equal(a[~na].view(ui), b[~nb].view(ui))
