"""The Viterbi transition matrix, restated here independently of the library.

The library and the CPU oracle both build the 13-state log-transition matrix
in hw_b200/csrc/hw_params.h.  This file restates the reference constructor
(Subframe::TransitionMatrix, src/basecaller/basecaller/traceAnalysis/
SubframeScorer.cpp:36-223, sparsity SubframeScorer.h:55-70) a second time, in
Python, keeping the reference's C++ types: the analog kinetics and the fudge
factors are float, computeLenProbs runs in double (frameRate is a double, so
`auto widthFrames = frameRate * widthSeconds` and everything after it is
double) and rounds to float on return, the matrix is filled in float and each
positive entry is replaced by std::log(float) (libm logf).  Both copies are
compared bit for bit at the reference defaults, the pinned workload
configuration, the kinetics of the reference's frame-labeler ground-truth
test (T/TestFrameLabeler.cpp:140-162, two-step pulse widths) and fudge
factors away from 1.
"""
import ctypes as C
import ctypes.util
import math

import numpy as np
import pytest

from hw_b200 import abi, native, workloads

f32 = np.float32
_libm = C.CDLL(ctypes.util.find_library("m"))
_libm.logf.argtypes = [C.c_float]
_libm.logf.restype = C.c_float
_libm.exp.argtypes = [C.c_double]
_libm.exp.restype = C.c_double

NA = 4
NS = 13


def _full(i):
    return 1 + i


def _up(i):
    return 1 + NA + i


def _down(i):
    return 1 + 2 * NA + i


def _len_probs(frame_rate, width_s, ratio):
    """computeLenProbs: double arithmetic, float results."""
    width_frames = float(frame_rate) * float(f32(width_s))
    ratio = max(f32(ratio), f32(1e-6))
    k1 = float(f32(1.0) + ratio) / width_frames
    k2 = float(f32(1.0) + f32(1.0) / ratio) / width_frames
    dk = k1 - k2
    c1 = float(f32(1.0)) - _libm.exp(-k1)
    c2 = float(f32(1.0)) - _libm.exp(-k2)
    r0 = 1 - k1 * c2 / k2 / dk + k2 * c1 / k1 / dk
    r1 = k1 * (c2 * c2) / k2 / dk - k2 * (c1 * c1) / k1 / dk
    r2 = k1 * (c2 * c2) * (1 - c2) / k2 / dk - k2 * (c1 * c1) * (1 - c1) / k1 / dk
    return [f32(r0), f32(r1), f32(r2)]


def _sparse_pattern():
    """(to, from) pairs the sparse matrix stores (SubframeScorer.h:55-70)."""
    cells = set()
    for r in range(NS):
        if r == 0 or 5 <= r <= 8:
            src = [0] + list(range(5, 13))
        elif 1 <= r <= 4:
            src = [r, r + 4]
        else:
            src = [r - 8, r - 4]
        cells |= {(r, c) for c in src}
    return cells


def reference_matrix(cfg):
    ipd = [f32(cfg.analogs[i].ipd_s) for i in range(NA)]
    pw = [f32(cfg.analogs[i].pulse_width_s) for i in range(NA)]
    ipd_r = [f32(cfg.analogs[i].ipd2_slow_step_ratio) for i in range(NA)]
    pw_r = [f32(cfg.analogs[i].pw2_slow_step_ratio) for i in range(NA)]
    delta = f32(0.01)
    for i in range(NA):
        # both tests read ipd2SlowStepRatio (SubframeScorer.cpp:58-74)
        if abs(ipd_r[i] - f32(1.0)) < delta:
            pw_r[i] = f32(1.0) - delta if pw_r[i] < f32(1.0) else f32(1.0) + delta
        if abs(ipd_r[i] - f32(1.0)) < delta:
            ipd_r[i] = f32(1.0) - delta if ipd_r[i] < f32(1.0) else f32(1.0) + delta
    s = f32(0.0)
    for i in range(NA):
        s = f32(s + ipd[i])
    mean_ipd = f32(s / f32(NA))
    fr = float(cfg.frame_rate)
    a_f, b_f, g_f = f32(cfg.viterbi_alpha), f32(cfg.viterbi_beta), f32(cfg.viterbi_gamma)

    ipd_len = [_len_probs(fr, ipd[i], ipd_r[i]) for i in range(NA)]
    alpha = [f32(f32(a_f * f32(0.25)) * f32(ipd_len[i][0] + ipd_len[i][1])) for i in range(NA)]
    alpha_sum = f32(0.0)
    for i in range(NA):
        alpha_sum = f32(alpha_sum + alpha[i])
    mean_len = _len_probs(fr, mean_ipd, f32(0.0))
    mean_ipd3m = f32(f32(f32(1.0) - mean_len[0]) - mean_len[1])
    start = f32(mean_len[2] / mean_ipd3m)

    d = np.zeros((NS, NS), np.float32)
    d[0, 0] = f32(1.0) - start
    for i in range(NA):
        full, up, down = _full(i), _up(i), _down(i)
        lp = _len_probs(fr, pw[i], pw_r[i])
        gamma = f32(f32(g_f * lp[0]) / f32(f32(1.0) + alpha_sum))
        beta = f32(b_f * lp[1])
        d[up, 0] = f32(0.25) * start
        d[0, up] = gamma
        d[down, up] = beta
        d[full, up] = f32(f32(f32(f32(1.0) - gamma) - f32(gamma * alpha_sum)) - beta)
        prob3ms = f32(f32(f32(1.0) - lp[0]) - lp[1])
        d[down, full] = f32(lp[2] / prob3ms)
        d[full, full] = f32(1.0) - d[down, full]
        d[0, down] = f32(1.0) - alpha_sum
        for j in range(NA):
            d[_up(j), down] = alpha[j]
            d[_up(j), up] = f32(gamma * alpha[j])

    # sparse storage: -inf off the pattern, 0 where the pattern holds a
    # non-positive probability (InitMatrix zero-fills), log elsewhere
    out = np.full((NS, NS), -np.inf, np.float32)
    for (r, c) in _sparse_pattern():
        out[r, c] = 0.0
    for r in range(NS):
        for c in range(NS):
            if d[r, c] > 0.0:
                out[r, c] = _libm.logf(float(d[r, c]))
    return out, d


def _labeler_test_movie():
    """Analog kinetics of the reference's frame-labeler ground-truth test."""
    cfg = workloads.chip_config()
    for i, (ipd, w) in enumerate(zip((.308, .234, .234, .188), (.232, .185, .181, .214))):
        cfg.analogs[i].ipd_s = ipd
        cfg.analogs[i].pulse_width_s = w
        cfg.analogs[i].ipd2_slow_step_ratio = 0.0
        cfg.analogs[i].pw2_slow_step_ratio = 3.2
    cfg.frame_rate = 100.0
    return cfg


def _configs():
    d = abi.Config()
    native.check(native.lib().hw_config_default(C.byref(d)))
    out = [("reference defaults", d), ("workload", workloads.chip_config()),
           ("labeler ground-truth movie", _labeler_test_movie())]
    c = _labeler_test_movie()
    c.viterbi_alpha, c.viterbi_beta, c.viterbi_gamma = 0.9, 1.1, 1.3
    out.append(("fudge factors 0.9/1.1/1.3", c))
    c = workloads.chip_config()
    c.analogs[1].ipd2_slow_step_ratio = 1.004      # inside the singularity guard
    c.analogs[1].pw2_slow_step_ratio = 0.5
    c.analogs[2].ipd2_slow_step_ratio = 2.5
    c.frame_rate = 80.0
    out.append(("ratios near 1, 80 fps", c))
    return out


@pytest.mark.parametrize("name,cfg", _configs(), ids=[n for n, _ in _configs()])
def test_library_matrix_equals_independent_restatement(name, cfg):
    want, probs = reference_matrix(cfg)
    # the probabilities of a proper kinetic model: every row of the
    # transposed matrix (the transitions out of a state) sums to ~1
    out_sums = probs.sum(axis=0)
    assert np.allclose(out_sums, 1.0, atol=1e-5), (name, out_sums)
    got = np.zeros((NS, NS), np.float32)
    native.check(native.lib().hw_transition_matrix(C.byref(cfg), abi.ptr(got)))
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (name, got, want)


@pytest.mark.parametrize("name,cfg", _configs(), ids=[n for n, _ in _configs()])
def test_oracle_matrix_equals_independent_restatement(name, cfg):
    import oracle
    want, _ = reference_matrix(cfg)
    got = oracle.transition_matrix(cfg)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), name


def test_restatement_known_structure():
    """Hand-checkable entries of the defaults: 0 -> up_i is a quarter of the
    pulse-start probability for every analog, and full -> full and
    full -> down are complementary."""
    _, d = reference_matrix(workloads.chip_config())
    ups = [d[_up(i), 0] for i in range(NA)]
    assert len(set(map(float, ups))) == 1
    assert math.isclose(float(ups[0]) * 4 + float(d[0, 0]), 1.0, rel_tol=1e-6)
    for i in range(NA):
        assert math.isclose(float(d[_full(i), _full(i)] + d[_down(i), _full(i)]), 1.0, rel_tol=1e-6)
