"""HF metrics (HFMetricsFilter): the oracle pinned by the reference's
known-answer test (T/TestHFMetricsFilter.cpp:300-430, `Populated`), and the
CUDA filter against the oracle bit for bit."""
import os

import numpy as np
import pytest

from hw_b200 import abi

HERE = os.path.dirname(os.path.abspath(__file__))
A, C, G, T = 0, 1, 2, 3          # Pulse::NucleotideLabel
MID = {G: 10, A: 20, T: 30, C: 40}
MAX = {G: 15, A: 25, T: 35, C: 45}
F, BLOCK, LANES, CAP = 512, 4096, 2, 48


def cart():
    return dict(np.load(os.path.join(HERE, "..", "hw_b200", "data", "trained_cart.npz")))


def fixed(v):
    """Pulse::ToFixedPrecision (DT/Pulse.h:210-216)."""
    return np.uint16(np.float32(v) / np.float32(0.1) + np.float32(0.5))


def sim_pulses(batch, pattern="ACGTGG", n=10, width=4, ipd=0):
    """GenerateBases of the reference test: n pulses per ZMW and batch."""
    lab = {"A": A, "C": C, "G": G, "T": T}
    p = np.zeros((LANES, abi.LANE, CAP), abi.PULSE_DT)
    lens = np.full((LANES, abi.LANE), n, np.uint32)
    for b in range(n):
        L = lab[pattern[b % len(pattern)]]
        mid = fixed(MID[L] + b)
        midf = np.float32(mid) * np.float32(0.1)
        mod = np.float32(1.1) if b % 2 == 0 else np.float32(1.01)
        rec = p[:, :, b]
        rec["start"] = b * width + b * ipd + batch * F
        rec["width"] = width
        rec["mid_signal"] = mid
        rec["mean_signal"] = mid
        rec["max_signal"] = fixed(MAX[L])
        rec["signal_m2"] = np.float32(np.float32(midf * midf) * np.float32(width - 2)) * mod
        rec["label"] = L
        rec["is_reject"] = 0
    return p, lens


def sim_inputs():
    """GenerateBaselineMetrics / FrameLabelerMetrics / PulseDetectorMetrics /
    Models of the reference test."""
    bs = np.zeros(LANES, abi.BLSTATS_DT)
    fa = bs["full_autocorr"]
    for k in range(4):
        fa["fbuf"][:, k, :] = -9.0 + 2 * k
        fa["bbuf"][:, k, :] = 6.0 + k
    fa["bidx"][:, 0, :] = min(F, 4)
    fa["bidx"][:, 1, :] = F % 4
    bs["raw_baseline_sum"] = 100
    bs["baseline_stats"]["moment0"] = 98
    bs["baseline_stats"]["moment1"] = 10
    bs["baseline_stats"]["moment2"] = 100
    fa["moment2"] = 2510
    fa["basic_stats"]["moment0"] = F
    fa["basic_stats"]["moment1"] = 110
    fa["basic_stats"]["moment2"] = 5650
    bs["background_stats"]["moment0"] = 42
    viterbi = np.full((LANES, abi.LANE), 1.09, np.float32)
    pd = np.zeros(LANES, abi.STAT_ACCUM_DT)
    pd["moment0"] = 98
    pd["moment1"] = 10
    pd["moment2"] = 100
    models = np.zeros(LANES, abi.LANE_MODEL_DT)
    for a, (m, v) in enumerate(zip((227.13, 154.45, 97.67, 61.32), (776, 426, 226, 132))):
        models["analogs"][:, a]["means"] = np.float16(m).view(np.uint16)
        models["analogs"][:, a]["vars"] = np.float16(v).view(np.uint16)
    models["baseline"]["means"] = np.float16(0).view(np.uint16)
    models["baseline"]["vars"] = np.float16(33).view(np.uint16)
    return bs, models, viterbi, pd


def check_populated(mb, pd):
    nb = BLOCK // F
    assert np.all(mb["num_pulse_frames"] == nb * 10 * 4)
    assert np.all(mb["num_base_frames"] == nb * 10 * 4)
    assert np.all(mb["num_half_sandwiches"] == nb * 8)
    assert np.all(mb["num_sandwiches"] == nb)
    assert np.all(mb["num_pulse_label_stutters"] == nb)
    for key in ("num_pulses_by_analog", "num_bases_by_analog", "num_pk_mid_bases_by_analog"):
        assert np.all(mb[key][:, A] == nb * 2) and np.all(mb[key][:, C] == nb * 2)
        assert np.all(mb[key][:, G] == nb * 4) and np.all(mb[key][:, T] == nb * 2)
    assert np.all(mb["num_pulses"] == nb * 10) and np.all(mb["num_bases"] == nb * 10)
    assert np.all(mb["activity_label"] == abi.HQRF_MULTI)
    assert np.all(mb["start_frame"] == 0) and np.all(mb["num_frames"] == nb * F)
    for a, v in zip((A, C, G, T), (736, 1408, 944, 1152)):
        assert np.all(mb["pk_mid_signal"][:, a] == v)
    for a, v in zip((A, C, G, T), (25, 45, 15, 35)):
        assert np.all(mb["pk_max"][:, a] == np.float32(fixed(v)) * np.float32(0.1))
    for a, v in zip((A, C, G, T), (0.0171916, 0.0043878, 0.0192236, 0.0065546)):
        assert np.all(np.abs(mb["bp_zvar"][:, a] - v) < 0.001)
    for a, v in zip((A, C, G, T), (0.0706076, 0.0451073, 0.0744171, 0.0960086)):
        assert np.all(np.abs(mb["pk_zvar"][:, a] - v) < 0.001)
    for a, n in zip((A, C, G, T), (2, 2, 4, 2)):
        assert np.all(mb["num_pk_mid_frames"][:, a] == nb * n * 2)
    assert np.all(np.abs(mb["autocorrelation"] - 0.415835) < 0.001)
    assert np.all(np.abs(mb["pulse_detection_score"] - 0.002128) < 0.0001)
    m0, m1, m2 = pd["moment0"], pd["moment1"], pd["moment2"]
    assert np.all(np.abs(mb["num_frames_baseline"] - m0 * nb) < 1e-4)
    assert np.all(np.abs(mb["frame_baseline_dws"] - m1 / m0) < 1e-4)
    assert np.all(np.abs(mb["frame_baseline_variance_dws"] - (m2 - m1 * m1 / m0) / (m0 - 1)) < 0.01)
    assert np.all(mb["pixel_checksum"] == 0)


def test_oracle_reproduces_reference_known_answers():
    import oracle
    bs, models, viterbi, pd = sim_inputs()
    hf = oracle.HfMetrics(LANES, BLOCK, 100.0, True)
    hf.set_cart(cart())
    got = []
    for batch in range(BLOCK // F):
        p, lens = sim_pulses(batch)
        got.append(hf.process(p, lens, bs, models, viterbi, pd, batch * F, F))
    assert all(g is None for g in got[:-1]) and got[-1] is not None
    check_populated(got[-1], pd)


def test_oracle_without_cart_labels_empty():
    import oracle
    bs, models, viterbi, pd = sim_inputs()
    hf = oracle.HfMetrics(LANES, BLOCK, 100.0, True)
    out = None
    for batch in range(BLOCK // F):
        p, lens = sim_pulses(batch)
        out = hf.process(p, lens, bs, models, viterbi, pd, batch * F, F)
    assert np.all(out["activity_label"] == abi.HQRF_EMPTY)
    assert np.all(out["num_pulses"] == 80)


def _equal_metrics(a, b):
    """Field-by-field equality; NaN == NaN (x86 and CUDA produce different NaN bits)."""
    for name in abi.BASECALLING_METRICS_DT.names:
        x, y = a[name], b[name]
        if x.dtype.kind == "f":
            if not np.array_equal(x, y, equal_nan=True):
                bad = np.argwhere(~((x == y) | (np.isnan(x) & np.isnan(y))))
                return f"{name} differs at {bad[:3].tolist()}: {x.flat[0]} vs {y.flat[0]}"
        elif not np.array_equal(x, y):
            return f"{name} differs"
    return None


@pytest.mark.gpu
def test_gpu_filter_matches_oracle_on_reference_case():
    import torch
    import oracle
    from hw_b200 import filters as Fl
    bs, models, viterbi, pd = sim_inputs()
    ref = oracle.HfMetrics(LANES, BLOCK, 100.0, True)
    ref.set_cart(cart())
    hf = Fl.HfMetrics(LANES, BLOCK, 100.0, True, cart=cart())
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a).view(np.uint8).reshape(-1).copy()).cuda()
    d_bs, d_models, d_vit, d_pd = dev(bs), dev(models), torch.from_numpy(viterbi).cuda(), dev(pd)
    for batch in range(BLOCK // F):
        p, lens = sim_pulses(batch)
        want = ref.process(p, lens, bs, models, viterbi, pd, batch * F, F)
        got = hf.process(dev(p), torch.from_numpy(lens).cuda(), CAP, d_bs, d_models, d_vit, d_pd, batch * F, F)
        assert (want is None) == (got is None)
    got = Fl.struct_to_numpy(got, abi.BASECALLING_METRICS_DT)
    check_populated(got, pd)
    assert _equal_metrics(got, want) is None, _equal_metrics(got, want)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [abi.DYNAMIC_ESTIMATIONS, abi.FIXED_ESTIMATIONS])
def test_gpu_filter_matches_oracle_on_chain_output(mode):
    """Pulses, statistics, Viterbi scores and models of the CUDA chain fed to
    the CUDA filter and to the oracle: identical metrics every block."""
    import torch
    import oracle
    import synth
    from hw_b200 import filters as Fl, workloads
    cfg = workloads.small_config()
    cfg.model_estimation_mode = mode
    lanes, Fc, chunks, block = 3, 512, 16, 1024
    tr = synth.traces(lanes, Fc * chunks, seed=7)
    an = Fl.BatchAnalyzer(cfg, 0, lanes, Fc)
    cap = cfg.max_calls_per_zmw
    hf = Fl.HfMetrics(lanes, block, cfg.frame_rate, True, cart=cart())
    ref = oracle.HfMetrics(lanes, block, cfg.frame_rate, True)
    ref.set_cart(cart())
    blocks = total = 0
    for c in range(chunks):
        chunk = torch.from_numpy(np.ascontiguousarray(tr[:, c * Fc:(c + 1) * Fc])).cuda()
        pulses, lens, ovf, em, est = an(chunk, c * Fc)
        if not em:
            continue
        bs, vit, pd = an.chunk_metrics()
        models, _ = an.models()
        first = c * Fc - abi.LATENT_FRAMES            # the labels batch (LabelsBatch.h:112-121)
        got = hf.process(pulses, lens, cap, bs, models, vit, pd, first, Fc)
        want = ref.process(Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(lanes, abi.LANE, cap),
                           lens.cpu().numpy().astype(np.uint32), Fl.struct_to_numpy(bs, abi.BLSTATS_DT),
                           Fl.struct_to_numpy(models, abi.LANE_MODEL_DT), vit.cpu().numpy(),
                           Fl.struct_to_numpy(pd, abi.STAT_ACCUM_DT), first, Fc)
        assert (got is None) == (want is None)
        if got is not None:
            blocks += 1
            g = Fl.struct_to_numpy(got, abi.BASECALLING_METRICS_DT)
            assert _equal_metrics(g, want) is None, _equal_metrics(g, want)
            total += int(g["num_pulses"].sum())
    assert blocks >= 2 and total > 0
