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


# The reference frame-labeler ground-truth test's movie (T/TestFrameLabeler.cpp:
# 140-181): kinetics of the four analogs (inter-pulse distance and pulse width
# in seconds, two-step pulse widths with ratio 3.2) and the fixed model it
# labels with (analog means and variances, baseline mean 0 and variance 33).
LABELER_TEST_IPD_S = (.308, .234, .234, .188)
LABELER_TEST_PW_S = (.232, .185, .181, .214)
LABELER_TEST_PW_RATIO = 3.2
LABELER_TEST_MEANS = (227.13, 154.45, 97.67, 61.32)
LABELER_TEST_VARS = (776.0, 426.0, 226.0, 132.0)
LABELER_TEST_BL_VAR = 33.0


def labeled_traces(lanes, frames, seed=0, frame_rate=100.0):
    """Baseline-subtracted traces with per-frame ground-truth labels, drawn
    from the labeler test's movie.  Pulses live in continuous time: analog
    uniform, pulse width the sum of two exponentials with the kinetic
    model's rates k1 = (1 + r) / w, k2 = (1 + 1 / r) / w (mean w frames), gap
    after a pulse exponential with the analog's mean inter-pulse distance.  A
    frame adds the analog mean and its excess variance times the fraction of
    the frame the pulse covers, over N(0, 33) baseline noise.  Ground truth
    (the labeler's state numbering: 0 baseline, 1 + a full, 5 + a up, 9 + a
    down): a pulse's first frame is up, its last frame (if it has two or
    more) is down, frames between are full.

    Returns (traces [lanes][frames][64] int16, truth [lanes][frames][64] int16)."""
    rng = np.random.default_rng(seed)
    n = lanes * 64
    sig = np.zeros((n, frames))
    extra = np.zeros((n, frames))
    truth = np.zeros((n, frames), np.int16)
    ipd = [d * frame_rate for d in LABELER_TEST_IPD_S]
    r = LABELER_TEST_PW_RATIO
    for z in range(n):
        t = rng.exponential(ipd[rng.integers(4)])
        while t < frames:
            a = int(rng.integers(4))
            w = LABELER_TEST_PW_S[a] * frame_rate
            width = rng.exponential(w / (1 + r)) + rng.exponential(w / (1 + 1 / r))
            start, end = t, t + width
            f0, f1 = int(start), int(np.ceil(end))
            for f in range(f0, min(f1, frames)):
                cover = min(end, f + 1) - max(start, f)
                sig[z, f] += LABELER_TEST_MEANS[a] * cover
                extra[z, f] += (LABELER_TEST_VARS[a] - LABELER_TEST_BL_VAR) * cover
            lab = np.full(f1 - f0, 1 + a, np.int16)
            lab[0] = 5 + a
            if f1 - f0 > 1:
                lab[-1] = 9 + a
            m = min(f1, frames) - f0
            truth[z, f0:f0 + m] = lab[:m]
            t = end + rng.exponential(ipd[a])
    tr = np.rint(sig + rng.standard_normal((n, frames)) * np.sqrt(LABELER_TEST_BL_VAR + extra))
    tr = np.clip(tr, -32768, 32767).astype(np.int16)
    to_lanes = lambda x: np.ascontiguousarray(x.reshape(lanes, 64, frames).transpose(0, 2, 1))
    return to_lanes(tr), to_lanes(truth)
