"""Preliminary HQ stage (PrelimHQFilterBody + the BazAggregator packet side):
the oracle pinned by the reference's PacketBufferManager and BazAggregator
tests (bazio/writing/test/TestPacketBufferManager.cpp,
TestBazAggregator.cpp) and the placeholder HQ rule of PrelimHQFilter.cpp;
the CUDA stage against the oracle byte for byte."""
import numpy as np
import pytest

from hw_b200 import abi

INTS = np.array([1, 2, 3, 4], np.int32).view(np.uint8)   # DummySerializer of the reference tests: 4 events, 16 bytes


def chunk(n, with_data):
    """One chunk's (bytes, offsets, events): the four ints for the ZMWs in with_data."""
    data, off, ev = [], np.zeros(n + 1, np.uint64), np.zeros(n, np.uint32)
    for z in range(n):
        if z in with_data:
            data.append(INTS)
            ev[z] = 4
        off[z + 1] = off[z] + (16 if z in with_data else 0)
    return (np.concatenate(data) if data else np.zeros(0, np.uint8)), off, ev


def marks(n, zs):
    m = np.zeros(n, np.uint8)
    m[list(zs)] = 1
    return m


def zmw(out, z):
    data, off, ev, hq = out
    return data[int(off[z]):int(off[z + 1])], int(ev[z])


def test_oracle_nothing_hq():
    """PacketBufferManager.ConstructNoHQ (TestPacketBufferManager.cpp:59-80)."""
    import oracle
    o = oracle.PrelimHq(10, 2, True)
    data, off, ev, hq = o.flush()
    assert len(data) == 0 and not ev.any() and not hq.any()


def test_oracle_add_data_mark_hq():
    """PacketBuffer.AddDataMarkHQ (:141-201): data of ZMWs not marked HQ is not
    returned; once marked, each returns its 4 events and 16 bytes."""
    import oracle
    o = oracle.PrelimHq(10, 1, True)
    o.add(*chunk(10, {0, 5}))
    data, off, ev, hq = o.flush()
    assert len(data) == 0 and not ev.any()
    out = o.end_block(marks(10, {0, 5}))
    for z in range(10):
        b, e = zmw(out, z)
        if z in (0, 5):
            assert e == 4 and b.tobytes() == INTS.tobytes()
        else:
            assert e == 0 and len(b) == 0
    assert out[3].sum() == 2


def test_oracle_lookback_buffers():
    """PacketBuffer.LookbackBuffers (:203-316): a ZMW marked HQ returns its
    data of every block in the window; one HQ before returns the block's."""
    import oracle
    o = oracle.PrelimHq(10, 3, True)
    o.add(*chunk(10, {0, 1, 2}))
    out = o.end_block(marks(10, {0}))
    assert out[3].sum() == 1 and zmw(out, 0)[1] == 4
    o.add(*chunk(10, {0, 1, 2}))
    out = o.end_block(marks(10, {1}))
    assert out[3].sum() == 2
    assert zmw(out, 0)[1] == 4 and zmw(out, 1)[1] == 8
    o.add(*chunk(10, {0, 1, 2}))
    out = o.end_block(marks(10, {2}))
    assert out[3].sum() == 3
    assert zmw(out, 0)[1] == 4 and zmw(out, 1)[1] == 4
    b, e = zmw(out, 2)
    assert e == 12 and b.view(np.int32).tolist() == [1, 2, 3, 4] * 3


def test_oracle_drops_data_past_the_window():
    """PacketBuffer.DropData (:318-344): ten blocks, a window of three."""
    import oracle
    o = oracle.PrelimHq(10, 3, True)
    for i in range(10):
        o.add(*chunk(10, {0}))
        out = o.end_block(marks(10, {0}) if i == 9 else np.zeros(10, np.uint8))
    b, e = zmw(out, 0)
    assert e == 12 and len(b) == 48


def placeholder(n, lookback, enable, stride, blocks):
    """DummyPreHQ::DetectHQ (PrelimHQFilter.cpp:173-206) by hand: the HQ set
    after each block."""
    hq = np.zeros(n, bool)
    seen = 0
    out = []
    for _ in range(blocks):
        if not enable:
            hq[:] = True
        else:
            seen += 1
            if seen >= lookback:
                pre = np.flatnonzero(~hq)
                hq[pre[::stride]] = True
        out.append(hq.copy())
    return out


@pytest.mark.parametrize("n,lookback,enable,throttle", [(12, 1, True, 1 / 3), (100, 3, True, 0.10),
                                                          (100, 3, False, 0.10), (37, 2, True, 0.25)])
def test_oracle_placeholder_rule(n, lookback, enable, throttle):
    """The placeholder HQ rule; (12, 1, 1/3) is BazAggregator.Iterators
    (TestBazAggregator.cpp:42-65): every third pre-HQ ZMW marked leaves 2/3."""
    import oracle
    o = oracle.PrelimHq(n, lookback, enable, throttle)
    stride = int(round(1 / np.float32(throttle)))
    want = placeholder(n, lookback, enable, stride, 6)
    for b in range(6):
        o.add(*chunk(n, set(range(n))))
        out = o.end_block()
        assert (out[3].astype(bool) == want[b]).all(), b
    if (n, lookback) == (12, 1):
        o2 = oracle.PrelimHq(n, 1, True, throttle)
        o2.add(*chunk(n, set(range(n))))
        assert (o2.end_block()[3] == 0).sum() == 2 * n // 3
        o2.add(*chunk(n, set(range(n))))
        assert (o2.end_block(np.ones(n, np.uint8))[3] == 0).sum() == 0


# ---- the CUDA stage ------------------------------------------------------------

def _run(n, cap, chunks_per_block, lookback, enable, throttle, blocks, seed, stride=1, mark_rate=None,
         which=abi.BAZ_PRODUCTION, extra_chunks=1):
    import torch
    import oracle
    from test_baz import preset, random_pulses
    from hw_b200 import filters as Fl
    f, skip = preset(which)
    gpu = Fl.PrelimHq(n, fields=f, skip_rejects=skip, chunks_per_block=chunks_per_block, lookback=lookback,
                      enable=enable, throttle=throttle, zmw_stride=stride)
    enc = oracle.BazEncoder(f, skip, n, zmw_stride=stride)
    ref = oracle.PrelimHq(n, lookback, enable, throttle)
    rng = np.random.default_rng(seed)
    nblocks = 0
    for c in range(blocks * chunks_per_block + extra_chunks):
        p, lens = random_pulses(rng, n, cap)
        data, off = enc(p, lens, cap)
        kept = np.minimum(lens, cap)[:, None] > np.arange(cap)[None, :]
        if skip:
            kept &= p["is_reject"] == 0
        kept[(np.arange(n) % 64) % stride != 0] = False
        ref.add(data, off, kept.sum(axis=1).astype(np.uint32))
        m = None
        if mark_rate is not None and (c + 1) % chunks_per_block == 0:
            m = (rng.random(n) < mark_rate).astype(np.uint8)
        d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
        d_l = torch.from_numpy(lens.view(np.int32)).cuda()
        got = gpu.process(d_p, d_l, cap, marks=None if m is None else torch.from_numpy(m).cuda())
        if (c + 1) % chunks_per_block:
            assert got is None
            continue
        want = ref.end_block(m)
        _same(got, want, n)
        assert got["block"] == nblocks
        nblocks += 1
    _same(gpu.flush(), ref.flush(), n)
    return nblocks


def _same(got, want, n):
    data, off, ev, hq = want
    assert got["offsets"].cpu().numpy().astype(np.uint64).tolist() == off.tolist()
    assert got["bytes"].cpu().numpy().tobytes() == data.tobytes()
    assert (got["events"].cpu().numpy() == ev).all()
    assert (got["hq"].cpu().numpy() == hq).all()
    assert got["num_hq"] == int(hq.sum())


@pytest.mark.gpu
def test_gpu_stage_placeholder_rule_matches_oracle():
    """Stride 4 (throttle 0.25), a window of three 3-chunk blocks, 7 blocks
    and an unfinished one flushed; ZMW bytes past the first slot sizes."""
    assert _run(700, 24, 3, 3, True, 0.25, 7, seed=1) == 7


@pytest.mark.gpu
def test_gpu_stage_preliminary_hq_off_matches_oracle():
    """enablePreHQ off: everything HQ at the first block."""
    assert _run(300, 16, 2, 10, False, 0.10, 4, seed=2, extra_chunks=0) == 4


@pytest.mark.gpu
@pytest.mark.parametrize("which", [abi.BAZ_PRODUCTION, abi.BAZ_INTERNAL])
def test_gpu_stage_caller_marks_and_stride_match_oracle(which):
    """The caller's HQ marks (20% a block), ZMW output stride 2, both encodings."""
    assert _run(500, 20, 2, 4, True, 0.10, 6, seed=3, stride=2, mark_rate=0.2, which=which) == 6


@pytest.mark.gpu
def test_gpu_stage_keeps_activity_labels():
    """MetricBufferManager::GetRecentActivityLabel: the labels of the last
    block's HF metrics; 4 (no label) before any."""
    import torch
    from test_baz import random_pulses
    from hw_b200 import filters as Fl
    n, cap = 256, 8
    st = Fl.PrelimHq(n, chunks_per_block=2, lookback=2)
    assert (st.activity().cpu().numpy() == 4).all()
    rng = np.random.default_rng(4)
    labels = rng.integers(0, 4, n).astype(np.uint8)
    metrics = np.zeros(n // abi.LANE, abi.BASECALLING_METRICS_DT)
    metrics["activity_label"] = labels.reshape(-1, abi.LANE)
    d_m = torch.from_numpy(metrics.view(np.uint8).reshape(-1).copy()).cuda()
    for c in range(2):
        p, lens = random_pulses(rng, n, cap)
        d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
        d_l = torch.from_numpy(lens.view(np.int32)).cuda()
        st.process(d_p, d_l, cap, metrics=d_m if c == 1 else None)
    assert (st.activity().cpu().numpy() == labels).all()
