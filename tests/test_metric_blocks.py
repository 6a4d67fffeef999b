"""The metric side of the preliminary HQ stage: the reference's metric-block
types (basecaller/dataTypes/Metrics.h) and MetricBufferManager
(bazio/writing/MetricBufferManager.h).

CPU: the oracle's half rounding against numpy's IEEE float16 (the `half`
2.1.0 library rounds to nearest even), the oracle against the reference's
own known-answer tests (basecaller/dataTypes/test/TestMetrics.cpp), the
manager on hand-worked schedules, and the oracle's reading of the two index
slips of MetricBufferManager.h (:263, :318).  GPU: the stage's metric
checkpoints (hw_prelim_hq_metrics) byte for byte against the oracle.
"""
import numpy as np
import pytest

from hw_b200 import abi
import oracle as O

LANE = abi.LANE


def hf_lanes(n_lanes, rng, labels=None, frames=4096):
    """One metric block of random HF metrics (abi.BASECALLING_METRICS_DT)."""
    m = np.zeros(n_lanes, abi.BASECALLING_METRICS_DT)
    L = (n_lanes, LANE)
    A = (n_lanes, abi.NUM_ANALOGS, LANE)
    m["activity_label"] = rng.integers(0, 4, L) if labels is None else labels.reshape(L)
    for f in ("num_pulse_frames", "num_base_frames", "num_sandwiches", "num_half_sandwiches",
              "num_pulse_label_stutters", "num_bases", "num_pulses"):
        m[f] = rng.integers(0, 3000, L)
    m["num_frames"] = frames - rng.integers(0, 3, L)
    m["num_frames_baseline"] = rng.choice([0, 1, 2, 700, 3100], L)
    m["frame_baseline_dws"] = rng.normal(0, 6, L).astype(np.float32)
    m["frame_baseline_variance_dws"] = rng.uniform(0, 90, L).astype(np.float32)
    m["num_pk_mid_frames"] = rng.choice([0, 1, 37, 400], A)
    m["pk_mid_signal"] = (rng.uniform(0, 400, A) * m["num_pk_mid_frames"]).astype(np.float32)
    m["num_pk_mid_bases_by_analog"] = rng.integers(0, 60, A)
    m["num_bases_by_analog"] = rng.integers(0, 900, A)
    m["pk_max"] = rng.uniform(-10, 70000, A).astype(np.float32)   # some past the half range
    m["bp_zvar"] = rng.uniform(0, 2, A).astype(np.float32)
    m["pk_zvar"] = rng.uniform(0, 9, A).astype(np.float32)
    m["autocorrelation"] = rng.uniform(-1, 1, L).astype(np.float32)
    m["pulse_detection_score"] = rng.normal(0, 30, L).astype(np.float32)
    return m


# ---- half rounding -------------------------------------------------------------

def test_half_rounding_equals_ieee_round_to_nearest_even():
    rng = np.random.default_rng(3)
    halves = np.arange(0, 0x7c00, dtype=np.uint16)
    hv = halves.view(np.float16).astype(np.float32)
    mids = ((hv[:-1].astype(np.float64) + hv[1:]) / 2).astype(np.float32)   # exact ties
    ulp = lambda x, k: (x.view(np.uint32).astype(np.int64) + k).astype(np.uint32).view(np.float32)
    x = np.concatenate([hv, mids, ulp(mids, 1), ulp(mids, -1), ulp(hv, 1), ulp(hv, -1),
                        np.ldexp(rng.uniform(1, 2, 200000), rng.integers(-30, 17, 200000)).astype(np.float32),
                        np.array([0, 65504, 65519.99, 65520, 1e30, np.inf, 2.0 ** -25, 2.0 ** -26], np.float32)])
    x = np.concatenate([x, -x])
    with np.errstate(over="ignore"):
        want = x.astype(np.float16).view(np.uint16)
    np.testing.assert_array_equal(O.half_bits(x), want)


def test_half_to_float_exact_for_every_half():
    bits = np.arange(0, 1 << 16, dtype=np.uint32).astype(np.uint16)
    finite = (bits & 0x7c00) != 0x7c00
    got = O.half_float(bits)
    want = bits.view(np.float16).astype(np.float32)
    np.testing.assert_array_equal(got[finite].view(np.uint32), want[finite].view(np.uint32))
    assert np.all(np.isinf(got[(bits & 0x7fff) == 0x7c00]))


# ---- the reference's known-answer tests (TestMetrics.cpp) -----------------------

def kat_lane():
    """MakeBasecallingMetrics (TestMetrics.cpp:32-58): every ZMW and analog
    alike; the fields the test leaves unset are 0."""
    m = np.zeros(1, abi.BASECALLING_METRICS_DT)
    m["activity_label"] = abi.HQRF_SINGLE
    m["num_pulse_frames"], m["num_base_frames"] = 100, 100
    m["num_sandwiches"], m["num_half_sandwiches"], m["num_pulse_label_stutters"] = 10, 20, 30
    m["num_bases"], m["num_pulses"] = 20, 30
    m["num_pk_mid_frames"] = 300
    m["pk_mid_signal"] = np.float32(238.18) * np.float32(300)
    m["bp_zvar"], m["pk_zvar"], m["pk_max"] = np.float32(3.32), np.float32(4.46), np.float32(347.9)
    m["num_pk_mid_bases_by_analog"] = 200
    m["frame_baseline_dws"], m["frame_baseline_variance_dws"] = 140.0, np.float32(35.9)
    m["num_frames_baseline"], m["num_frames"] = 200, 4096
    m["autocorrelation"], m["pulse_detection_score"] = np.float32(10.32), np.float32(5.6)
    return m


def float_eq(a, b):
    """gtest EXPECT_FLOAT_EQ: within 4 units in the last place."""
    a, b = np.float32(a), np.float32(b)
    ia, ib = (int(v.view(np.int32)) for v in (a, b))
    ia = ia if ia >= 0 else -(ia & 0x7fffffff)
    ib = ib if ib >= 0 else -(ib & 0x7fffffff)
    return abs(ia - ib) <= 4


def test_kat_production():
    bm = kat_lane()
    # ProductionMetrics<uint32_t, float>{bm, 0} aggregating {bm, 1}
    sm, raw = O.metrics_kat(bm, 0)
    nf, pw, bw, npul, nb, nbf, npf0, mean, var = raw[:9]
    assert (nf, pw, bw, npul, nb) == (4096 * 2, 200, 200, 60, 40)
    assert float_eq(np.float32(238.18) * np.float32(300) * 2, np.float32(raw[9]) * np.float32(npf0))
    assert npf0 == 600 and nbf == 400
    assert float_eq(140.0, mean) and float_eq(np.float32(35.9), var)
    assert sm["activity_label"] == abi.HQRF_SINGLE
    # an empty ProductionMetrics<uint32_t, float> aggregating the half-precision block once, then ten times
    want = np.float32(238.18) * np.float32(300) / np.float32(300)
    for reps in (1, 10):
        _, raw = O.metrics_kat(bm, 1, reps=reps)
        assert np.isfinite(raw[9] * raw[6])
        assert abs(want - raw[9]) <= 0.1


def test_kat_aggregate():
    bm = kat_lane()
    sm, raw = O.metrics_kat(bm, 2)
    single = O.metric_block(bm, 0, "production_float")
    assert raw[0] == 2 * single["num_frames"] and raw[1] == 2 * single["pulse_width"]
    assert raw[2] == 2 * single["base_width"] and raw[3] == 2 * single["num_pulses"]
    assert raw[4] == 2 * 20
    assert float_eq(single["pkmid"][3], raw[10])
    assert float_eq(np.float32(35.9), raw[8])
    assert raw[6] == 2 * single["num_pkmid_frames"][1] and raw[5] == 2 * single["num_baseline_frames"]


def test_kat_complete():
    bm = kat_lane()
    sm, raw = O.metrics_kat(bm, 3)
    ns, nhs, nst, pds, tac, pkmax0, npb0, pkz0, bpz0 = raw[11:20]
    assert (ns, nhs, nst) == (20, 40, 60)
    assert float_eq(np.float32(5.6), pds) and float_eq(np.float32(10.32), tac)
    assert float_eq(np.float32(347.9), pkmax0) and npb0 == 400
    assert float_eq(np.float32(4.46), pkz0) and float_eq(np.float32(3.32), bpz0)
    # the converted counts go through the uint16_t setters
    assert sm["num_sandwiches"] == 20 and sm["num_pkmid_bases"][0] == 400


def test_conversion_of_one_block_by_type():
    """Field by field: counts as given, values rounded to half where the type
    is half, the baseline sd the half sqrt of the half variance."""
    rng = np.random.default_rng(5)
    lane = hf_lanes(1, rng)
    h = lambda v: O.half_float(O.half_bits(np.float32(v)))
    for z in (0, 17, 63):
        p = O.metric_block(lane, z, "production_half")
        c = O.metric_block(lane, z, "complete_half")
        m = lane[0]
        assert p["num_frames"] == m["num_frames"][z] and p["activity_label"] == m["activity_label"][z]
        assert p["baseline"] == h(m["frame_baseline_dws"][z])
        assert p["baseline_sd"] == h(np.sqrt(h(m["frame_baseline_variance_dws"][z])))
        for a in range(4):
            n = m["num_pk_mid_frames"][a][z]
            want = h(np.float32(m["pk_mid_signal"][a][z]) / np.float32(n)) if n else 0.0
            assert p["pkmid"][a] == want
            assert c["pkmax"][a] == h(m["pk_max"][a][z]) and c["pkzvar"][a] == h(m["pk_zvar"][a][z])
        assert p["pulse_detection_score"] == 0 and c["pulse_detection_score"] == h(m["pulse_detection_score"][z])
        assert c["num_half_sandwiches"] == m["num_half_sandwiches"][z]


# ---- the manager ---------------------------------------------------------------

def scripted(n_lanes, n_zmw, block, labels):
    """Metrics whose counts say where they came from: num_frames =
    100 + 10 * block + z, labels as given (per ZMW)."""
    m = np.zeros(n_lanes, abi.BASECALLING_METRICS_DT)
    z = np.arange(n_lanes * LANE)
    m["num_frames"] = (100 + 10 * block + z).reshape(n_lanes, LANE)
    lab = np.zeros(n_lanes * LANE, np.uint8)
    lab[:n_zmw] = labels
    m["activity_label"] = lab.reshape(n_lanes, LANE)
    m["num_frames_baseline"] = 50
    m["frame_baseline_dws"], m["frame_baseline_variance_dws"] = 10.0, 4.0
    return m


def frames_and_labels(blocks, off, n):
    return [[(int(b["num_frames"]), int(b["activity_label"])) for b in blocks[off[z]:off[z + 1]]] for z in range(n)]


@pytest.mark.parametrize("literal", [False, True])
def test_manager_hand_worked_schedule(literal):
    """Four ZMWs, a window of three blocks, ZMW 1 marked HQ at block 3 with
    labels 0,1,1,2,2,3 over blocks 0..5 (the others keep label 0)."""
    ms = O.MetricSide(4, 3, True, literal=literal)
    lab1 = [0, 1, 1, 2, 2, 3]
    got = []
    for b in range(6):
        ms.add(scripted(1, 4, b, [0, lab1[b], 0, 0]))
        newly = np.array([0, 1 if b == 3 else 0, 0, 0], np.uint8)
        got.append(frames_and_labels(*ms.end_block(newly), 4))
    got.append(frames_and_labels(*ms.flush(), 4))
    empty = [[], [], [], []]
    assert got[0] == got[1] == got[2] == got[4] == empty
    # block 3: ZMW 1's pre-HQ aggregate (block 0), then the run of blocks 1-2
    # (label 1); block 3 (label 2) stays open
    assert got[3] == [[], [(101, 0), (111 + 121, 1)], [], []]
    # block 4 joins the open run; block 5's label change emits it
    assert got[5] == [[], [(131 + 141, 2)], [], []]
    # flush: ZMW 1's open run; the others their pre-HQ aggregates of blocks 0..3
    assert got[6] == [[(460, 0)], [(151, 3)], [(468, 0)], [(472, 0)]]


def test_manager_index_slip_of_the_reference():
    """A window of one block, ZMW 0 marked at block 0 and ZMW 1 at block 1:
    ZMW 1's window index is then 0, and the reference aggregates its later
    blocks into ZMW 0's open aggregate (MetricBufferManager.h:263)."""
    outs = {}
    for literal in (False, True):
        ms = O.MetricSide(2, 1, True, literal=literal)
        seq = []
        for b in range(4):
            ms.add(scripted(1, 2, b, [1, 1]))
            seq.append(frames_and_labels(*ms.end_block(np.array([b == 0, b == 1], np.uint8)), 2))
        seq.append(frames_and_labels(*ms.flush(), 2))
        outs[literal] = seq
    # block 0: ZMW 0's empty pre-HQ aggregate; block 1: ZMW 1's (its block 0)
    for lit in (False, True):
        assert outs[lit][0] == [[(0, 4)], []] and outs[lit][1] == [[], [(101, 1)]]
    # each ZMW's own blocks: 0 -> 100+110+120+130, 1 -> 111+121+131
    assert outs[False][4] == [[(460, 1)], [(363, 1)]]
    # the reference: ZMW 1's blocks 2 and 3 land in ZMW 0's aggregate
    assert outs[True][4] == [[(460 + 121 + 131, 1)], [(111, 1)]]


def run_schedule(ms, n, lanes, blocks, marks, seed):
    rng = np.random.default_rng(seed)
    lab = rng.integers(0, 4, n)
    out = []
    for b in range(blocks):
        flip = rng.random(n) < 0.35
        lab = np.where(flip, rng.integers(0, 4, n), lab)
        full = np.zeros(lanes * LANE, np.uint8)
        full[:n] = lab
        ms.add(hf_lanes(lanes, np.random.default_rng(seed * 1000 + b), labels=full))
        blk, off = ms.end_block(marks(b))
        out.append((blk.view(np.uint8).copy(), off.copy()))
    blk, off = ms.flush()
    out.append((blk.view(np.uint8).copy(), off.copy()))
    return out


def test_literal_equals_own_entries_while_the_slips_are_no_ops():
    """Marking from the highest ZMW down (no ZMW below a marked one is ever
    HQ before it) keeps both slips no-ops: the reference's reading and the
    stage's agree byte for byte over 24 blocks."""
    n, lanes, W = 150, 3, 4
    order = np.arange(n)[::-1]

    def marks(b):
        m = np.zeros(n, np.uint8)
        m[order[b * 7:(b + 1) * 7]] = 1
        return m

    a = run_schedule(O.MetricSide(n, W, True, literal=False), n, lanes, 24, marks, 11)
    b = run_schedule(O.MetricSide(n, W, True, literal=True), n, lanes, 24, marks, 11)
    assert sum(int(o[-1]) for _, o in a) > 200
    for (xa, oa), (xb, ob) in zip(a, b):
        np.testing.assert_array_equal(oa, ob)
        np.testing.assert_array_equal(xa, xb)


def test_complete_metrics_one_block_per_zmw_per_block():
    n, lanes = 150, 3
    for stride in (1, 4):
        ms = O.MetricSide(n, 10, False, zmw_stride=stride)
        rng = np.random.default_rng(stride)
        for b in range(3):
            lane = hf_lanes(lanes, rng)
            ms.add(lane)
            blk, off = ms.end_block(np.ones(n, np.uint8))
            cnt = np.diff(off.astype(np.int64))
            np.testing.assert_array_equal(cnt, (np.arange(n) % stride == 0).astype(np.int64))
            for z in range(0, n, stride):
                want = O.metric_block(lane[z // LANE:z // LANE + 1], z % LANE, "complete_half")
                assert blk[off[z]].tobytes() == want.tobytes()
        assert len(ms.flush()[0]) == 0


# ---- GPU: the stage against the oracle ------------------------------------------

def _stage_run(n, lanes, W, cpb, enable, stride, blocks, seed, marks_fn=None, metric_chunks=None):
    import torch
    from hw_b200 import filters as Fl
    stage = Fl.PrelimHq(n, chunks_per_block=cpb, lookback=W, enable=enable, throttle=0.25, zmw_stride=stride,
                        metrics=True)
    om = O.MetricSide(n, W, enable, zmw_stride=stride)
    op = O.PrelimHq(n, W, enable, 0.25)
    cap = 4
    pulses = torch.zeros(n * cap * abi.PULSE_DT.itemsize, dtype=torch.uint8, device="cuda")
    lens = torch.zeros(n, dtype=torch.int32, device="cuda")
    rng = np.random.default_rng(seed)
    lab = rng.integers(0, 4, n)
    hq_prev = np.zeros(n, np.uint8)
    checked = 0
    for b in range(blocks):
        flip = rng.random(n) < 0.3
        lab = np.where(flip, rng.integers(0, 4, n), lab)
        full = np.zeros(lanes * LANE, np.uint8)
        full[:n] = lab
        hf = hf_lanes(lanes, np.random.default_rng(seed * 977 + b), labels=full)
        dev_hf = torch.from_numpy(hf.view(np.uint8).copy()).cuda()
        marks = None if marks_fn is None else marks_fn(b)
        dev_marks = None if marks is None else torch.from_numpy(marks).cuda()
        at = cpb - 1 if metric_chunks is None else metric_chunks(b)
        cp = None
        for c in range(cpb):
            cp = stage.process(pulses, lens, cap, metrics=dev_hf if c == at else None,
                               marks=dev_marks if c == cpb - 1 else None)
        om.add(hf)
        op.add(np.zeros(0, np.uint8), np.zeros(n + 1, np.uint64), np.zeros(n, np.uint32))
        _, _, _, hq = op.end_block(marks)
        want, woff = om.end_block((hq != 0) & (hq_prev == 0))
        hq_prev = hq
        torch.cuda.synchronize()
        np.testing.assert_array_equal(cp["hq"].cpu().numpy(), hq)
        mc = stage.metric_checkpoint()
        np.testing.assert_array_equal(mc["offsets"].cpu().numpy().astype(np.uint64), woff, err_msg=f"block {b}")
        got = mc["blocks"].cpu().numpy()
        assert got.tobytes() == want.view(np.uint8).tobytes(), f"block {b}"
        assert mc["block"] == b
        checked += len(want)
    stage.flush()
    want, woff = om.flush()
    mc = stage.metric_checkpoint()
    np.testing.assert_array_equal(mc["offsets"].cpu().numpy().astype(np.uint64), woff)
    assert mc["blocks"].cpu().numpy().tobytes() == want.view(np.uint8).tobytes()
    np.testing.assert_array_equal(stage.activity().cpu().numpy(), om.activity())
    return checked + len(want)


@pytest.mark.gpu
@pytest.mark.parametrize("W,cpb,stride", [(3, 2, 1), (1, 1, 1), (5, 3, 2)])
def test_gpu_production_metrics_equal_oracle(W, cpb, stride):
    """Preliminary HQ on, the placeholder rule marking every 4th pre-HQ ZMW
    from block W-1 on, 20 blocks of random metrics (runs of labels, counts
    past 16 bits once aggregated, values past the half range)."""
    assert _stage_run(1000, 16, W, cpb, True, stride, 20, seed=W * 10 + cpb) > 1000


@pytest.mark.gpu
def test_gpu_production_metrics_caller_marks_and_mid_block_metrics():
    n, rng = 333, np.random.default_rng(8)

    def marks(b):
        return (rng.random(n) < 0.08).astype(np.uint8)

    assert _stage_run(n, 6, 4, 3, True, 1, 14, seed=4, marks_fn=marks, metric_chunks=lambda b: b % 3) > 100


@pytest.mark.gpu
@pytest.mark.parametrize("stride", [1, 8])
def test_gpu_complete_metrics_equal_oracle(stride):
    assert _stage_run(700, 11, 10, 2, False, stride, 4, seed=stride) > 0
