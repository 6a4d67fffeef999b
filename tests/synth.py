"""Seeded synthetic traces for the tests (numpy, host side).

Per ZMW: a 200 DN baseline with N(0, 8^2) noise; pulses from four analogs of
80/50/32/20 DN (uniform choice, 10% amplitude CV per pulse); a pulse starts on
a baseline frame with probability 1/ipd and ends after each pulse frame with
probability 1/width, so widths and gaps are geometric with means 8 and 14
frames; pulse frames get shot-noise variance 0.5 x amplitude on top of the
baseline variance.  Options add a lognormal per-ZMW gain, empty ZMWs and a
baseline random walk.  Output layout is [lanes][frames][64] int16.
"""
import numpy as np

AMPS = np.array([80.0, 50.0, 32.0, 20.0])


def traces(lanes, frames, seed=0, width=8.0, ipd=14.0, gain_sigma=0.0, empty_fraction=0.0,
           walk_sigma=0.0, baseline=200.0, sigma=8.0, amp_cv=0.1, shot=0.5):
    rng = np.random.default_rng(seed)
    n = lanes * 64
    gain = np.exp(gain_sigma * rng.standard_normal(n)) if gain_sigma > 0 else np.ones(n)
    empty = rng.random(n) < empty_fraction
    out = np.empty((frames, n), np.float64)
    inp = np.zeros(n, bool)
    amp = np.zeros(n)
    walk = np.zeros(n)
    for t in range(frames):
        u = rng.random(n)
        start = (~inp) & (~empty) & (u < 1.0 / ipd)
        end = inp & (u < 1.0 / width)
        a = AMPS[rng.integers(0, 4, n)] * (1.0 + amp_cv * rng.standard_normal(n)) * gain
        amp = np.where(start, np.maximum(a, 0.0), amp)
        inp = np.where(start, True, np.where(end, False, inp))
        sig = np.where(inp, amp, 0.0)
        if walk_sigma > 0:
            walk += walk_sigma * rng.standard_normal(n)
        out[t] = baseline + walk + sig + rng.standard_normal(n) * np.sqrt(sigma * sigma + shot * sig)
    tr = np.clip(np.rint(out), -32768, 32767).astype(np.int16)
    return np.ascontiguousarray(tr.reshape(frames, lanes, 64).transpose(1, 0, 2))
