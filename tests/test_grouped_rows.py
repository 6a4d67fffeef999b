"""The labeler's grouped 9-way Viterbi rows, restated in float32 numpy and
checked against the generic rows on adversarial inputs: exact ties, ties
after rounding (a later state whose log-likelihood is a few ulps below the
group's largest), -inf groups and mixtures.  The grouped rows either return
the generic rows' value and traceback code or flag the frame for the generic
rows (the rounding check), never a different answer.  The transition
constants are the reference's at its defaults, where each 9-way row's
constants are equal within the source groups 5..8 and 9..12."""
import numpy as np

import oracle
from hw_b200 import workloads

F32 = np.float32
NINF = F32(-np.inf)
ROWS = (0, 5, 6, 7, 8)
SOURCES = (0, 5, 6, 7, 8, 9, 10, 11, 12)


def generic_row(T, R, score, ll):
    """Candidates (score + T[R][s]) + ll[s] in source order; ties go to the
    later source (the labeler's Pick)."""
    mv, win = None, None
    for s in SOURCES:
        v = F32(F32(score + T[R, s]) + ll[s])
        if mv is None or v >= mv:
            mv, win = v, s
    return mv, win


def scan_group(vals):
    """The largest value, its last position and the largest after it (NaN
    when it is the group's last position), right to left."""
    m, pos, after = vals[3], 3, F32(np.nan)
    for p in (2, 1, 0):
        if vals[p] > m:
            after, m, pos = m, vals[p], p
    return m, pos, after


def grouped_row(T, R, score, ll, gA, gB):
    """The grouped row: returns (value, winner, slow)."""
    c0 = F32(F32(score + T[R, 0]) + ll[0])
    aA, aB = F32(score + T[R, 5]), F32(score + T[R, 9])
    (mA, pA, afA), (mB, pB, afB) = gA, gB
    gvA, gvB = F32(aA + mA), F32(aB + mB)
    nvA, nvB = F32(aA + afA), F32(aB + afB)
    geA = gvA >= c0
    mv = gvA if geA else c0
    geB = gvB >= mv
    if geB:
        return gvB, 9 + pB, bool(nvB == gvB)
    if geA:
        return mv, 5 + pA, bool(nvA == gvA)
    return mv, 0, False


def _frames(rng, n):
    """log-likelihood vectors with the situations that matter."""
    out = []
    for _ in range(n):
        base = F32(rng.uniform(-3000.0, -10.0))
        ll = (base + rng.normal(0, 5, 13)).astype(F32)
        kind = rng.integers(0, 6)
        if kind == 1:       # exact ties inside the groups
            ll[6] = ll[5]
            ll[11] = ll[9]
        elif kind == 2:     # a later state a few ulps below the group's largest
            for g in (5, 9):
                p = g + rng.integers(0, 3)
                q = p + 1 + rng.integers(0, g + 3 - p)
                ll[q] = np.nextafter(ll[p], NINF, dtype=F32)
                for _ in range(rng.integers(0, 4)):
                    ll[q] = np.nextafter(ll[q], NINF, dtype=F32)
                if ll[q] > max(ll[g:g + 4][ll[g:g + 4] != ll[q]], default=NINF):
                    ll[p] = np.nextafter(ll[q], F32(np.inf), dtype=F32)
        elif kind == 3:     # a group of -inf (non-ROI frames)
            ll[5:9] = NINF
        elif kind == 4:     # every state but the baseline -inf
            ll[1:] = NINF
        elif kind == 5:     # large magnitudes: coarse ulps, many rounding ties
            ll = (F32(-2.0e6) + rng.integers(-3, 4, 13).astype(F32)).astype(F32)
        out.append(ll)
    return out


def test_grouped_rows_equal_generic_rows_or_flag_them():
    T = oracle.transition_matrix(workloads.chip_config()).astype(F32)
    for R in ROWS:
        assert (T[R, 5:9] == T[R, 5]).all() and (T[R, 9:13] == T[R, 9]).all()
    rng = np.random.default_rng(7)
    flagged = checked = 0
    for ll in _frames(rng, 4000):
        gA, gB = scan_group(ll[5:9]), scan_group(ll[9:13])
        for R in ROWS:
            score = F32(rng.uniform(-40.0, 0.0))
            v0, w0 = generic_row(T, R, score, ll)
            v1, w1, slow = grouped_row(T, R, score, ll, gA, gB)
            if slow:
                flagged += 1
                continue
            checked += 1
            assert v1.tobytes() == v0.tobytes() and w1 == w0, (R, ll, score)
    # the adversarial frames reach the rounding check, and most rows pass it
    assert flagged > 0 and checked > 10 * flagged
