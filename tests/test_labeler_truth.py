"""Frame labels against synthetic ground truth, mirroring the reference's
CompareVsGroundTruth test (src/basecaller/basecaller/test/
TestFrameLabeler.cpp:104-251).

The reference test labels a simulated SNR-40 trace file (missing from the
reference checkout) with a fixed model and the movie's kinetics, then
classifies every labelled frame against the file's ground truth: equal
labels are matches; unequal ones where either label is a sub-frame state
(up or down, > 4) are sub-frame confusions; the rest are mismatches.  It
requires matches > 97%, sub-frame confusions < 2% and mismatches < 1%.

Here the traces come from tests/synth.py:labeled_traces, drawn from the same
movie (analog kinetics with two-step pulse widths, the test's fixed model:
analog means 227.13 / 154.45 / 97.67 / 61.32, variances 776 / 426 / 226 /
132, baseline 0 with variance 33) with sub-frame pulse starts and ends, and
the same layout: 2 pools of 2 lanes, 64 chunks of 128 frames, labels lagging
the chunk by the 24 latent frames.  The oracle's labeler must meet the
reference's thresholds; a shifted truth or swapped analog means must not
(the check has teeth).  On the GPU the library's labeler must produce the
oracle's labels, latent traces and Viterbi scores bit for bit and so meet
the same thresholds.
"""
import numpy as np
import pytest

import synth
from hw_b200 import abi, workloads

LANES_PER_POOL, POOLS = 2, 2
BLOCK_LEN, N_BLOCKS = 128, 64
LATENT = abi.LATENT_FRAMES


def movie_config():
    cfg = workloads.chip_config()
    for i in range(4):
        cfg.analogs[i].ipd_s = synth.LABELER_TEST_IPD_S[i]
        cfg.analogs[i].pulse_width_s = synth.LABELER_TEST_PW_S[i]
        cfg.analogs[i].ipd2_slow_step_ratio = 0.0
        cfg.analogs[i].pw2_slow_step_ratio = synth.LABELER_TEST_PW_RATIO
    cfg.frame_rate = 100.0
    return cfg


def fixed_model(lanes, means=synth.LABELER_TEST_MEANS):
    h = lambda x: np.float16(x).view(np.uint16)
    m = np.zeros(lanes, abi.LANE_MODEL_DT)
    m["baseline"]["means"] = h(0.0)
    m["baseline"]["vars"] = h(synth.LABELER_TEST_BL_VAR)
    m["baseline"]["weights"] = h(0.5)
    for i in range(4):
        m["analogs"][:, i]["means"] = h(means[i])
        m["analogs"][:, i]["vars"] = h(synth.LABELER_TEST_VARS[i])
        m["analogs"][:, i]["weights"] = h(0.125)
    return m


class OracleLabeler:
    def __init__(self, cfg, pool_id, lanes, margin=False):
        import oracle
        self.p = oracle.Pool(cfg, lanes, BLOCK_LEN, pool_id)
        self.margin = margin

    def __call__(self, chunk, models):
        return self.p.label(chunk, models, self.margin)


class GpuLabeler:
    def __init__(self, cfg, pool_id, lanes, margin=False):
        import torch
        from hw_b200 import filters as Fl
        self.torch, self.Fl = torch, Fl
        self.lab = Fl.FrameLabeler(cfg, pool_id, lanes, BLOCK_LEN)
        self.margin = margin

    def __call__(self, chunk, models):
        out = self.lab(self.torch.from_numpy(chunk).cuda(), self.Fl.numpy_to_struct(models), self.margin)
        self.torch.cuda.synchronize()
        return tuple(t.cpu().numpy() for t in out)


def run(make, traces, means=synth.LABELER_TEST_MEANS, margin=False):
    """Label every chunk of every pool; returns the per-chunk outputs."""
    cfg = movie_config()
    out = []
    for p in range(POOLS):
        lab = make(cfg, p, LANES_PER_POOL, margin)
        models = fixed_model(LANES_PER_POOL, means)
        tr = traces[p * LANES_PER_POOL:(p + 1) * LANES_PER_POOL]
        out.append([lab(np.ascontiguousarray(tr[:, c * BLOCK_LEN:(c + 1) * BLOCK_LEN]), models)
                    for c in range(tr.shape[1] // BLOCK_LEN)])
    return out


def score(outputs, truth, shift=0):
    """LabelValidator counts (TestFrameLabeler.cpp:200-205): labels batch
    frame j of a chunk starting at frame c * 128 is trace frame c * 128 + j -
    24; frames before 0 are skipped."""
    matches = sub = mism = 0
    nf = truth.shape[1]
    for p, chunks in enumerate(outputs):
        t = truth[p * LANES_PER_POOL:(p + 1) * LANES_PER_POOL]
        for c, res in enumerate(chunks):
            labels = res[0]
            for j in range(BLOCK_LEN):
                frame = c * BLOCK_LEN + j - LATENT + shift
                if frame < 0 or frame >= nf:
                    continue
                a, e = labels[:, j, :], t[:, frame, :]
                eq = a == e
                sf = ~eq & ((a > 4) | (e > 4))
                matches += int(eq.sum())
                sub += int(sf.sum())
                mism += int((~eq & ~sf).sum())
    total = matches + sub + mism
    return matches / total, sub / total, mism / total


@pytest.fixture(scope="module")
def data():
    return synth.labeled_traces(LANES_PER_POOL * POOLS, BLOCK_LEN * N_BLOCKS, seed=40)


@pytest.fixture(scope="module")
def oracle_out(data):
    return run(OracleLabeler, data[0], margin=True)


def agree_except_small_margin(a, b, margin, tol=1e-5):
    """The parity rule for labels: equal except where the decision that
    chose the label was closer than `tol`."""
    return bool(np.all((a == b) | (margin < tol)))


def test_oracle_meets_reference_thresholds(data, oracle_out):
    m, s, x = score(oracle_out, data[1])
    assert m > 0.97 and s < 0.02 and x < 0.01, (m, s, x)


def test_oracle_margins(oracle_out):
    """Margins are gaps between the winning and the next candidate: never
    negative or NaN; the last label's is a probability gap in [0, 1]
    (up to rounding);
    the margin option leaves labels, latent traces and scores unchanged."""
    for chunks in oracle_out:
        for labels, lat, score, mg in chunks:
            assert not np.isnan(mg).any() and (mg >= 0).all()
            assert (mg[:, -1, :] <= np.float32(1 + 1e-6)).all()     # normalised in float: may round above 1
    import oracle
    cfg = movie_config()
    a = oracle.Pool(cfg, 1, BLOCK_LEN)
    b = oracle.Pool(cfg, 1, BLOCK_LEN)
    tr, _ = synth.labeled_traces(1, BLOCK_LEN * 4, seed=3)
    m = fixed_model(1)
    for c in range(4):
        chunk = np.ascontiguousarray(tr[:, c * BLOCK_LEN:(c + 1) * BLOCK_LEN])
        ra, rb = a.label(chunk, m), b.label(chunk, m, True)
        for x, y in zip(ra, rb[:3]):
            assert np.array_equal(x.view(np.uint8), y.view(np.uint8))


def test_thresholds_catch_a_shifted_truth(data, oracle_out):
    m, s, x = score(oracle_out, data[1], shift=1)
    assert not (m > 0.97 and s < 0.02 and x < 0.01), (m, s, x)


def test_thresholds_catch_swapped_analogs(data):
    means = list(synth.LABELER_TEST_MEANS)
    means[0], means[1] = means[1], means[0]
    out = run(OracleLabeler, data[0][:, :BLOCK_LEN * 16], means)
    m, s, x = score(out, data[1][:, :BLOCK_LEN * 16])
    assert not (m > 0.97 and s < 0.02 and x < 0.01), (m, s, x)


@pytest.mark.gpu
def test_gpu_labels_equal_oracle_and_meet_thresholds(data, oracle_out):
    got = run(GpuLabeler, data[0])
    for p in range(POOLS):
        for c in range(N_BLOCKS):
            for k, what in enumerate(("labels", "latent", "viterbi score")):
                a, b = got[p][c][k], oracle_out[p][c][k]
                assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8)), (p, c, what)
    m, s, x = score(got, data[1])
    assert m > 0.97 and s < 0.02 and x < 0.01, (m, s, x)


@pytest.mark.gpu
def test_gpu_margins_equal_oracle(data, oracle_out):
    """hw_labeler_process with a margin buffer: labels, latent traces,
    scores and every label's margin equal the oracle's bit for bit, so the
    rule 'labels equal except where the margin is under 1e-5' can be
    evaluated at the C ABI."""
    got = run(GpuLabeler, data[0], margin=True)
    for p in range(POOLS):
        for c in range(N_BLOCKS):
            for k, what in enumerate(("labels", "latent", "viterbi score", "margin")):
                a, b = got[p][c][k], oracle_out[p][c][k]
                assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8)), (p, c, what)
            assert agree_except_small_margin(got[p][c][0], oracle_out[p][c][0], oracle_out[p][c][3])
