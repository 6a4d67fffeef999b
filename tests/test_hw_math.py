"""The shared arithmetic of the chain (hw_b200/csrc/hw_math.h), through the
oracle build of the same header: Cephes-method exp/log accuracy against
double precision, float->fp16 rounding against numpy, and the reference's
float->int16 conversion rule (cvtps2dq round-to-nearest-even, NaN and
out-of-range to INT32_MIN, then the low 16 bits; common/simd/m512f_SSE.h:
126-131 and m512s_SSE.h:101-110)."""
import numpy as np
import pytest

import oracle


def _ulp_err(got, exact):
    got = np.float32(got)
    ref = np.float32(exact)
    if ref == 0:
        return 0 if got == 0 else np.inf
    return abs(float(got) - exact) / float(np.spacing(np.abs(ref)))


def test_expf_accuracy():
    rng = np.random.default_rng(0)
    xs = np.concatenate([rng.uniform(-87.0, 88.0, 4000), np.linspace(-10, 10, 2001), [0.0, -0.0, 1.0, -1.0]])
    worst = max(_ulp_err(oracle.expf(x), np.exp(np.float64(np.float32(x)))) for x in xs)
    assert worst <= 2.0, worst


def test_expf_limits():
    assert oracle.expf(0.0) == 1.0
    assert oracle.expf(-104.0) == 0.0
    assert oracle.expf(89.0) == np.inf
    assert np.isnan(oracle.expf(np.nan))
    # IEEE-like denormal results between -103.97 and -87.3
    v = oracle.expf(-100.0)
    assert 0 < v < np.finfo(np.float32).tiny


def test_logf_accuracy():
    rng = np.random.default_rng(1)
    xs = np.concatenate([np.exp(rng.uniform(-80, 80, 4000)), np.linspace(0.5, 2.0, 1001)])
    worst = max(_ulp_err(oracle.logf(x), np.log(np.float64(np.float32(x)))) for x in xs)
    assert worst <= 2.0, worst


def test_logf_limits():
    assert oracle.logf(1.0) == 0.0
    assert oracle.logf(0.0) == -np.inf
    assert np.isnan(oracle.logf(-1.0))
    assert oracle.logf(np.inf) == np.inf


def test_f16_rounding_matches_numpy():
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.standard_normal(3000).astype(np.float32) * 300,
                         rng.uniform(-70000, 70000, 1000).astype(np.float32),
                         np.float32([0.0, -0.0, 65504.0, 65520.0, 1e-8, 6e-8, np.inf, -np.inf])])
    L = oracle.lib()
    got = np.array([L.or_f32_to_f16(float(x)) for x in xs], np.uint16)
    assert np.array_equal(got, xs.astype(np.float16).view(np.uint16))


def _cvt_i16_reference(x):
    x = np.float32(x)
    if np.isnan(x) or x >= 2147483648.0 or x < -2147483648.0:
        r = -2147483648
    else:
        r = int(np.rint(np.float64(x)))     # round half to even
    return np.int16(np.int64(r) & 0xFFFF if (np.int64(r) & 0xFFFF) < 0x8000 else (np.int64(r) & 0xFFFF) - 0x10000)


@pytest.mark.parametrize("x", [0.5, 1.5, 2.5, -0.5, -1.5, 32767.4, 32767.5, 32768.0, -32768.6, 65535.0, 70000.3,
                               -70000.7, 1e10, -1e10, np.nan, np.inf, -np.inf, 123.456])
def test_float_to_int16_rule(x):
    assert oracle.lib().or_to_i16(float(x)) == _cvt_i16_reference(x)
