"""Known-answer tests of the CPU oracle, restated from the reference's own
unit tests (test inputs and expected values re-derived from the test
sources; no reference code runs here).

* trace histogram: basecaller/test/TestTraceHistogramAccumulator.cpp:318-925
  (ResetFromStats, SingleLane/MultiLane/MultiPool constant, Sawtooth
  simple/skip/outliers/outliers-stagger, Reset);
* pulse accumulator accept/reject sweep:
  basecaller/test/TestPulseAccumulator.cpp:366-590;
* window (extremum) filter sawtooth:
  prototypes/BaselineFilter/test/testExtremaFilter.cu:20-125;
* detection-model EM on a simulated five-mode mixture:
  basecaller/test/TestDmeEm.cpp:158-456 (SNR sweep, 5-sigma tolerances,
  the reference test's own std::mt19937(42) draws).

The synthetic signals follow appModules/SimulatedDataSource.cpp:42-250: a
cache of ceil(numSignals/64) lanes is filled from the generator and lane i of
any pool reads cache lane i % numLanes.
"""
import numpy as np
import pytest

import oracle
from hw_b200 import abi, workloads

NB = abi.NUM_BINS
LANE = abi.LANE


# ---- SimulatedDataSource generators ---------------------------------------

def constant_signal(num_frames, idx):
    """ConstantGenerator (SimulatedDataSource.h:155-167): value = signal index."""
    return np.full(num_frames, idx, np.int16)


def sawtooth_signal(num_frames, idx, min_amp, max_amp, period, stagger):
    """SawtoothGenerator::GenerateSignal (SimulatedDataSource.cpp:237-250)."""
    rng = max_amp - min_amp + 1
    slope = float(rng) / period
    out = np.empty(num_frames, np.int16)
    for i in range(num_frames):
        v = int(slope * (i + idx * stagger))          # static_cast<int16_t>(double), truncation
        out[i] = min_amp + (v % rng)
    return out


def pool_traces(gen, num_signals, lanes_per_pool, pool, num_frames):
    """[lanes][frames][64] int16 for one pool, replicating the cache lanes."""
    cache_lanes = (num_signals + LANE - 1) // LANE
    out = np.empty((lanes_per_pool, num_frames, LANE), np.int16)
    for l in range(lanes_per_pool):
        cl = (pool * lanes_per_pool + l) % cache_lanes
        for z in range(LANE):
            out[l, :, z] = gen(num_frames, cl * LANE + z)
    return out


def mock_models(lanes, bl_mean=0.0, bl_var=1.0):
    m = np.zeros(lanes, abi.LANE_MODEL_DT)
    m["baseline"]["means"][:] = abi.f32_to_f16(bl_mean)
    m["baseline"]["vars"][:] = abi.f32_to_f16(bl_var)
    return m


def run_histograms(lanes_per_pool, pools, F, num_frames, lo, hi, gen, num_signals):
    """Reset(bounds) then AddBatch per chunk, as Histogram::RunTest does."""
    cfg = workloads.small_config()
    out = []
    for p in range(pools):
        pool = oracle.Pool(cfg, lanes_per_pool, F, p)
        b = np.zeros(lanes_per_pool, abi.HIST_BOUNDS_DT)
        b["lower_bounds"][:] = lo
        b["upper_bounds"][:] = hi
        pool.hist_reset_from_bounds(b)
        tr = pool_traces(gen, num_signals, lanes_per_pool, p, num_frames)
        models = mock_models(lanes_per_pool)
        for c in range(num_frames // F):
            pool.hist_add(tr[:, c * F:(c + 1) * F], (c * F, (c + 1) * F), models)
        h, fi = pool.hist_get()
        out.append((pool, h, fi))
    return out


# ---- Trace histogram -------------------------------------------------------

def test_histogram_reset_from_stats():
    """TestTraceHistogramAccumulator.cpp:318-364."""
    cfg = workloads.small_config()
    lanes = 2
    pool = oracle.Pool(cfg, lanes, 512, 1)
    st = np.zeros(lanes, abi.BLSTATS_DT)
    for l in range(lanes):
        t = np.arange(LANE, dtype=np.float32) + l * LANE + 2
        bs = st[l]["baseline_stats"]
        bs["offset"][:] = 0
        bs["moment0"][:] = t
        bs["moment1"][:] = t * t
        bs["moment2"][:] = 2 * t * t * t
    pool.hist_reset_from_stats(st)
    h, fi = pool.hist_get()
    assert fi == (0, 0)
    for l in range(lanes):
        for z in range(LANE):
            frames = np.float32(z + l * LANE + 2)
            mean = frames
            if frames >= cfg.baseline_stat_min_frame_count:
                sig = np.sqrt(mean * mean * mean / (mean - np.float32(1)), dtype=np.float32)
            else:
                sig = np.float32(cfg.fallback_baseline_sigma)
            expect = np.float32(cfg.bin_size_coeff) * sig
            # EXPECT_FLOAT_EQ: within 4 ulp
            assert abs(int(np.float32(h[l]["bin_size"][z]).view(np.int32)) - int(expect.view(np.int32))) <= 4
            assert h[l]["low_bound"][z] < mean - 2 * sig


@pytest.mark.parametrize("case", ["single_lane", "multi_lane", "multi_pool"])
def test_histogram_constant(case):
    """SingleLaneConstant / MultiLaneConstant / MultiPoolConstant
    (TestTraceHistogramAccumulator.cpp:366-500): bin = signal index, the
    edge-frame filter drops the first and last frame."""
    lanes, pools = {"single_lane": (1, 1), "multi_lane": (4, 1), "multi_pool": (2, 2)}[case]
    num_signals = LANE if case == "single_lane" else lanes * pools * LANE
    res = run_histograms(lanes, pools, 512, 2048, 0.0, float(NB), constant_signal, num_signals)
    for p, (_, h, fi) in enumerate(res):
        assert fi == (0, 2048)
        for l in range(lanes):
            assert not h[l]["outlier_count_low"].any() and not h[l]["outlier_count_high"].any()
            expected = np.zeros((NB, LANE), np.uint16)
            base = ((p * lanes + l) % ((num_signals + LANE - 1) // LANE)) * LANE
            for z in range(LANE):
                expected[base + z, z] = 2048 - 2
            assert np.array_equal(h[l]["bin_count"], expected)


def test_histogram_sawtooth_simple_uniform():
    """TestTraceHistogramAccumulator.cpp:502-581: bins 0, 1, 2 and 299 are all
    edge frames; every other bin holds 6 or 7 counts."""
    gen = lambda n, i: sawtooth_signal(n, i, 0, NB, NB, 0)
    for _, h, fi in run_histograms(2, 2, 512, 2048, 0.0, float(NB), gen, LANE):
        assert fi == (0, 2048)
        for l in range(2):
            assert not h[l]["outlier_count_low"].any() and not h[l]["outlier_count_high"].any()
            c = h[l]["bin_count"]
            for i in range(NB):
                if i in (0, 1, 2, NB - 1):
                    assert not c[i].any(), i
                else:
                    assert np.isin(c[i], (6, 7)).all(), (i, c[i])


def test_histogram_sawtooth_skip_uniform():
    """TestTraceHistogramAccumulator.cpp:583-643: even values only; bins 2 and
    298 are edge frames."""
    period = NB // 2
    gen = lambda n, i: sawtooth_signal(n, i, 0, NB, period, 0)
    expect = 2048 // period
    for _, h, _ in run_histograms(2, 2, 512, 2048, 0.0, float(NB), gen, LANE):
        for l in range(2):
            assert not h[l]["outlier_count_low"].any() and not h[l]["outlier_count_high"].any()
            c = h[l]["bin_count"]
            for i in range(NB):
                if i in (2, NB - 2) or i % 2 == 1:
                    assert not c[i].any(), i
                else:
                    assert np.isin(c[i], (expect, expect + 1)).all(), (i, c[i])


def test_histogram_sawtooth_outliers_uniform():
    """TestTraceHistogramAccumulator.cpp:645-724: range [100, 400), values
    0..511 four times; 4 counts per bin, 511 high edge frames."""
    gen = lambda n, i: sawtooth_signal(n, i, 0, 512, 512, 0)
    for _, h, _ in run_histograms(2, 2, 512, 2048, 100.0, 100.0 + NB, gen, LANE):
        for l in range(2):
            assert (h[l]["outlier_count_high"] == 4 * (512 - (100 + NB) - 1)).all()
            assert (h[l]["outlier_count_low"] == 4 * (100 - 0 - 3)).all()
            assert (h[l]["bin_count"] == 4).all()


def test_histogram_sawtooth_outliers_stagger():
    """TestTraceHistogramAccumulator.cpp:726-840: ZMW z starts 2z into the
    ramp; the first and last frames of each ZMW are edge frames too."""
    periods, period, lo, hi = 4, 512, 100, 100 + NB
    gen = lambda n, i: sawtooth_signal(n, i, 0, period, period, 2)
    z = np.arange(LANE, dtype=np.int32)
    first = z * 2
    last = (first + periods * period - 1) % period
    edge_hi = periods + ((first < period - 1) & (first >= hi)) + ((last < period - 1) & (last >= hi))
    exp_hi = (period - hi) * periods - edge_hi
    edge_lo = 3 * periods + ((first > 2) & (first < lo)) + ((last > 2) & (last < lo))
    exp_lo = (lo - 0) * periods - edge_lo
    for _, h, _ in run_histograms(2, 2, period, periods * period, float(lo), float(hi), gen, LANE):
        for l in range(2):
            assert np.array_equal(h[l]["outlier_count_high"].astype(np.int32), exp_hi)
            assert np.array_equal(h[l]["outlier_count_low"].astype(np.int32), exp_lo)
            for i in range(NB):
                v = i + lo
                expect = 4 - (first == v).astype(np.int32) - (last == v).astype(np.int32)
                assert np.array_equal(h[l]["bin_count"][i].astype(np.int32), expect), i


def test_histogram_reset():
    """TestTraceHistogramAccumulator.cpp:842-925: after Reset(bounds 5..10)
    the histogram is empty with the new binning."""
    gen = lambda n, i: sawtooth_signal(n, i, 0, 512, 512, 2)
    for pool, h, _ in run_histograms(2, 2, 512, 2048, 100.0, 100.0 + NB, gen, LANE):
        for l in range(2):
            assert (h[l]["outlier_count_high"] > 0).all() and (h[l]["outlier_count_low"] > 0).all()
            assert (h[l]["bin_count"] > 0).all()
        b = np.zeros(2, abi.HIST_BOUNDS_DT)
        b["lower_bounds"][:] = 5
        b["upper_bounds"][:] = 10
        pool.hist_reset_from_bounds(b)
        h2, fi = pool.hist_get()
        assert fi == (0, 0)
        for l in range(2):
            assert not h2[l]["outlier_count_high"].any() and not h2[l]["outlier_count_low"].any()
            assert (h2[l]["low_bound"] == np.float32(5)).all()
            assert (h2[l]["bin_size"] == np.float32(5) / np.float32(NB)).all()
            assert not h2[l]["bin_count"].any()


# ---- Pulse accumulator -----------------------------------------------------

KEEP = [  # ampThresh, widThresh, ipd, width  (TestPulseAccumulator.cpp:555-569)
    (0.999, 16.0, 24, 40), (0.999, 44.0, 8, 56), (0.999, 58.0, 4, 60), (0.999, 61.0, 2, 62),
    (0.999, 63.0, 1, 63), (12.0 / (1 + 12.1), 50.0, 40, 24), (24.0 / (1 + 24.1), 50.0, 40, 24),
    (40.0 / (1 + 40.1), 16.0, 24, 40)]
REJECT = [  # TestPulseAccumulator.cpp:571-580
    (0.999, 64.0, 1, 63), (0.999, 40.0, 32, 32), (36.0 / (1 + 36.1), 50.0, 52, 12)]


@pytest.mark.parametrize("amp_thresh, wid_thresh, ipd, pw, keep",
                         [k + (True,) for k in KEEP] + [r + (False,) for r in REJECT])
def test_pulse_accumulator_accept_reject(amp_thresh, wid_thresh, ipd, pw, keep):
    """TestPulseAccumulatorRejection::RunTest (TestPulseAccumulator.cpp:406-548)
    with this build's 24 latent frames: a fixed pattern of `ipd` baseline
    frames and a pulse of width `pw` (up state, full states, down state) of
    analog base % 4 at a constant 60 + 20 * (base % 4)."""
    cfg = workloads.small_config()
    cfg.xsp_amp_thresh = np.float32(amp_thresh)
    cfg.xsp_width_thresh = np.float32(wid_thresh)
    F, L, first = 512, abi.LATENT_FRAMES, 512
    assert F % (ipd + pw) == 0
    rng = np.random.default_rng(1)
    labels, trace = [], []
    base, frame = 0, first - L
    while frame < first + F - L:
        trace += list(np.round(rng.normal(0.0, 10.0, ipd)).astype(np.int16))
        labels += [0] * ipd + [base % 4 + 5] + [base % 4 + 1] * (pw - 2) + [base % 4 + 9]
        trace += [60 + ((frame + L) // (ipd + pw)) % 4 * 20] * pw
        frame += ipd + pw
        base += 1
    expected_count = base - 1          # the last pulse ends at the chunk boundary
    lab = np.repeat(np.asarray(labels, np.int16)[:, None], LANE, 1)[None]
    tr = np.repeat(np.asarray(trace, np.int16)[:, None], LANE, 1)[None]
    latent = np.ascontiguousarray(tr[:, :L])
    cur = np.zeros((1, F, LANE), np.int16)
    cur[:, :F - L] = tr[:, L:]
    models = np.zeros(1, abi.LANE_MODEL_DT)
    for a in range(4):
        models[0]["analogs"][a]["means"][:] = abi.f32_to_f16(20.0 * (6 - a))
    pool = oracle.Pool(cfg, 1, F)
    pulses, lens, ovf, _ = pool.pulses(lab, latent, cur, first - L, models)
    assert (lens == expected_count).all() and not ovf.any()
    for z in (0, 37, 63):
        for n in range(expected_count):
            p = pulses[0, z, n]
            pi = n % 4
            amp = 20.0 * (6 - (4 - pi - 1))
            assert bool(p["is_reject"]) == (not keep)
            assert p["label"] == pi                       # analogs A, C, G, T
            assert p["start"] == first - L + n * (ipd + pw) + ipd
            assert p["width"] == pw
            assert p["mean_signal"] == round(amp * 10) and p["max_signal"] == round(amp * 10)
            assert p["mid_signal"] == round(amp * 10)
            assert abs(p["signal_m2"] - amp * amp * (pw - 2)) <= amp


# ---- Window (extremum) filter ----------------------------------------------

def test_extremum_filter_sawtooth():
    """testExtremaFilter.cu:20-107: a width-7 max filter over a height-25
    sawtooth in 64-frame blocks; from frame 7 on the output is the previous
    frame's value, or the ramp top while the top is inside the window."""
    W, H, F, frames = 7, 25, 64, 256
    sig = sawtooth_signal(frames, 0, 0, H, H, 0)
    blocks = np.repeat(sig.reshape(frames // F, F)[:, :, None], LANE, 2)
    out = oracle.extremum_stage(W, True, blocks).reshape(frames, LANE)
    for t in range(W, frames):
        e = (t - 1) % H
        if e < W - 1:
            e = H - 1
        assert (out[t] == e).all(), t


@pytest.mark.parametrize("W", [3, 7, 11, 17, 61])
@pytest.mark.parametrize("is_max", [True, False])
def test_extremum_filter_matches_sliding_window(W, is_max):
    """Output m is the extremum of inputs m-W .. m-1, with W zeros before the
    first input (TraceFilters.cpp:11-57 on a WindowBuffer that starts with
    W zeros), across block boundaries."""
    rng = np.random.default_rng(W)
    F, chunks = 64, 5
    x = rng.integers(-32768, 32767, size=(chunks * F, LANE), dtype=np.int16)
    out = oracle.extremum_stage(W, is_max, x.reshape(chunks, F, LANE)).reshape(chunks * F, LANE)
    padded = np.concatenate([np.zeros((W, LANE), np.int16), x])
    op = np.max if is_max else np.min
    ref = np.stack([op(padded[m:m + W], axis=0) for m in range(chunks * F)])
    assert np.array_equal(out, ref)


# ---- Detection-model EM ----------------------------------------------------

def _dme_config():
    """TestDmeEm SetUp (TestDmeEm.cpp:404-430): refSnr 5, 80 fps,
    photoelectron sensitivity 2, relative amplitudes 3.70/2.55/1.68/1.0 and
    the shot-variance coefficient the test asserts (1.2168207), no pulse
    amplitude regularisation and model update method 0.  The mock movie's
    excess-noise CV is not in the reference sources; 0.1 (the value of the
    reference's mock dye set, MockExperimentData.cpp:58) is used."""
    cfg = workloads.small_config()
    cfg.ref_snr = 5.0
    cfg.frame_rate = 80.0
    cfg.photoelectron_sensitivity = 2.0
    cfg.shot_var_coeff = np.float32(1.2168207)
    cfg.pulse_amp_regularization = 0.0       # TestDmeEm() json (TestDmeEm.cpp:131-137)
    cfg.model_update_method = 0
    for a, ra in enumerate((3.70, 2.55, 1.68, 1.0)):
        cfg.analogs[a].rel_amplitude = ra
    return cfg


def _stats_for(bl_weight_frames, total, mean, var):
    """Baseliner stats whose baseline mode has the given count/mean/variance."""
    st = np.zeros(1, abi.BLSTATS_DT)
    bs = st[0]["baseline_stats"]
    n = np.float32(bl_weight_frames)
    bs["moment0"][:] = n
    bs["moment1"][:] = np.float32(mean) * n
    bs["moment2"][:] = np.float32(var) * (n - 1) + np.float32(mean) * np.float32(mean) * n
    st[0]["full_autocorr"]["basic_stats"]["moment0"][:] = np.float32(total)
    return st


class _Mt19937NormalFloat:
    """std::mt19937(seed) feeding libstdc++'s std::normal_distribution<float>
    (Marsaglia polar method; generate_canonical<float, 24> takes one 32-bit
    draw: float(u) / 2^32, with 1.0 replaced by the float below it).  numpy's
    MT19937 with legacy seeding is the same engine as std::mt19937; logf and
    sqrtf come from the C library as in the reference build."""

    def __init__(self, seed):
        import ctypes
        self.bg = np.random.MT19937(0)
        self.bg._legacy_seeding(seed)
        libm = ctypes.CDLL("libm.so.6")
        libm.logf.restype = ctypes.c_float
        libm.logf.argtypes = [ctypes.c_float]
        self.logf = libm.logf
        self.saved = None

    def _canonical(self):
        u = np.float32(int(self.bg.random_raw()))
        r = np.float32(u / np.float32(4294967296.0))
        return r if r < 1 else np.nextafter(np.float32(1), np.float32(0))

    def __call__(self):
        if self.saved is not None:
            v, self.saved = self.saved, None
            return v
        while True:
            x = np.float32(float(np.float32(2) * self._canonical()) - 1.0)
            y = np.float32(float(np.float32(2) * self._canonical()) - 1.0)
            r2 = np.float32(x * x + y * y)
            if not (r2 > 1.0 or r2 == 0.0):
                break
        mult = np.sqrt(np.float32(np.float32(-2) * np.float32(self.logf(float(r2)))) / r2, dtype=np.float32)
        self.saved = np.float32(x * mult)
        return np.float32(y * mult)


@pytest.mark.parametrize("sim_snr", [3.6, 4.0, 5.0, 6.0])
def test_dme_em_snr_sweep(sim_snr):
    """TestDmeEm EstimateFiniteMixture (TestDmeEm.cpp:158-243, 271-388,
    449-456) with the reference test's own random inputs: frames {500, 125,
    125, 125, 125} of analogs 0..3 then baseline, one std::mt19937(42) normal
    draw per frame shared by all 64 ZMWs, drawn from the start model
    InitLaneDetModel(0.5, 0, 100) rescaled to `sim_snr` (ScaleModelSnr,
    DmeEmHost.cpp:837-852).  Every estimated mixture fraction, mean and
    variance must lie within 5 sigma of the complete-data value."""
    cfg = _dme_config()
    n_frames = (500, 125, 125, 125, 125)
    total = sum(n_frames)
    pool = oracle.Pool(cfg, 1, 1024)     # the histogram takes any frame count
    # InitLaneDetModel(0.5, 0, 100) through the stats path: baseline weight
    # 101/202, mean 0, variance 100 (fp16 model, confidence 0 = initModelConf).
    start = pool.init_models(_stats_for(101, 202, 0.0, 100.0))
    start["confidence"][:] = abi.f32_to_f16(0.0)
    # the simulation model: float copy of the start model, analog means scaled
    # by simSnr / refSnr and variances from ModelSignalCovar.
    f = np.float32(np.float32(sim_snr) / np.float32(cfg.ref_snr))
    bl_var = abi.f16_to_f32(start["baseline"]["vars"][0, 0])
    means = [abi.f16_to_f32(start["baseline"]["means"][0, 0])]
    sds = [np.sqrt(bl_var, dtype=np.float32)]
    for a in range(4):
        m = np.float32(f * abi.f16_to_f32(start["analogs"][0][a]["means"][0]))
        cv2 = np.float32(cfg.analogs[a].excess_noise_cv) ** 2
        v = np.float32(np.float32(bl_var + np.float32(cfg.shot_var_coeff) * m) + np.float32(cv2 * np.float32(m * m)))
        means.append(m)
        sds.append(np.sqrt(v, dtype=np.float32))
    gauss = _Mt19937NormalFloat(42)
    x = np.empty(total, np.float32)
    mode = np.empty(total, np.int32)
    t = 0
    for m in (1, 2, 3, 4, 0):                    # analogs first, then baseline
        for _ in range(n_frames[m]):
            x[t] = np.floor(np.float32(sds[m] * gauss() + means[m]))
            mode[t] = m
            t += 1
    traces = np.repeat(x.astype(np.int16)[:, None], LANE, 1)[None]
    # BaselinerStatAccumulator over the trace (baseline frames flagged)
    st = np.zeros(1, abi.BLSTATS_DT)
    m0 = m1 = m2 = np.float32(0)
    for v in x[mode == 0]:
        m0, m1, m2 = np.float32(m0 + 1), np.float32(m1 + v), np.float32(m2 + v * v)
    bs = st[0]["baseline_stats"]
    bs["moment0"][:], bs["moment1"][:], bs["moment2"][:] = m0, m1, m2
    st[0]["full_autocorr"]["basic_stats"]["moment0"][:] = np.float32(total)
    pool.hist_reset_from_stats(st)
    pool.hist_add(traces, (0, total), start)
    hist, hfi = pool.hist_get()
    models, diag = pool.estimate(hist, st, hfi, (0, total), start)
    res = models[0]
    assert (abi.f16_to_f32(res["confidence"]) > 0).all(), "estimation failed"
    for m in range(5):
        sel = x[mode == m]
        w = np.float32(n_frames[m]) / np.float32(total)
        s1 = np.float32(0)
        for v in sel:
            s1 = np.float32(s1 + v)
        cd_mean = np.float32(s1 / np.float32(len(sel)))
        s2 = np.float32(0)
        for v in sel:
            s2 = np.float32(s2 + np.float32(v - cd_mean) ** 2)
        cd_var = np.float32(s2 / np.float32(len(sel) - 1))
        src = res["baseline"] if m == 0 else res["analogs"][m - 1]
        r_w = abi.f16_to_f32(src["weights"])
        r_mean = abi.f16_to_f32(src["means"])
        r_var = abi.f16_to_f32(src["vars"])
        tol_w = 5 * np.sqrt(w * (1 - w) / total)
        if m > 0:
            tol_w = max(np.float32(0.015), tol_w)
        assert (np.abs(r_w - w) <= tol_w).all(), (m, r_w[0], w)
        tol_m = 5 * np.sqrt(cd_var / total / w)
        assert (np.abs(r_mean - cd_mean) <= tol_m).all(), (m, r_mean[0], cd_mean, tol_m)
        tol_v = 5 * np.sqrt(2.0 / (total * w - 1)) * cd_var
        assert (np.abs(r_var - cd_var) <= tol_v).all(), (m, r_var[0], cd_var, tol_v)


def test_static_model_restates_setup_analogs():
    """FixedModelBatchAnalyzer's model (BatchAnalyzer.cpp:119-144) from
    StaticDetModelConfig::SetupAnalogs (StaticDetModelConfig.h:53-68), in float
    arithmetic and stored as fp16."""
    cfg = workloads.small_config()
    cfg.static_baseline_mean = 3.0
    cfg.static_baseline_variance = 33.0
    m = oracle.static_model(cfg, 2)
    f32 = np.float32
    bl_mean, bl_var = f32(3.0), f32(33.0)
    ref_signal = f32(f32(cfg.ref_snr) * np.sqrt(bl_var, dtype=np.float32))
    assert (m["baseline"]["means"] == abi.f32_to_f16(bl_mean)).all()
    assert (m["baseline"]["vars"] == abi.f32_to_f16(bl_var)).all()
    for a in range(4):
        mean = f32(bl_mean + f32(f32(cfg.analogs[a].rel_amplitude) * ref_signal))
        cm = f32(f32(cfg.analogs[a].excess_noise_cv) * mean)
        var = f32(f32(bl_var + mean) + f32(cm * cm))
        assert (m["analogs"][:, a]["means"] == abi.f32_to_f16(mean)).all()
        assert (m["analogs"][:, a]["vars"] == abi.f32_to_f16(var)).all()
    assert not m["confidence"].any() and not m["analogs"]["weights"].any()
