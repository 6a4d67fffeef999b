"""BAZ pulse encoding (bazio/encoding): the oracle pinned by the reference's
known-answer tests (bazio/encoding/test/TestFieldSerializers.cpp,
TestFieldTransforms.cpp, TestPulseToBaz.cu, TestBazRoundTrip.cpp), and the
CUDA encoder against the oracle byte for byte."""
import ctypes as C

import numpy as np
import pytest

from hw_b200 import abi

M64 = 2**64 - 1
A, Cc, G, T = 0, 1, 2, 3


def s64(u):
    """uint64 as a signed integer."""
    return u - 2**64 if u >= 2**63 else u


def field(name, transform=abi.BAZ_NOOP, serialize=abi.BAZ_TRUNCATE, bits=7, signed=False, scale=0, tbytes=0,
          ovbytes=0):
    f = np.zeros(1, abi.BAZ_FIELD_DT)[0]
    f["name"], f["store_signed"], f["transform"], f["scale"] = name, int(signed), transform, scale
    f["transform_bytes"], f["serialize"], f["num_bits"], f["overflow_bytes"] = tbytes, serialize, bits, ovbytes
    return f


def fields(*fs):
    return np.array(list(fs), abi.BAZ_FIELD_DT)


def kestrel(width_ser, ovbytes=0):
    """Label / PulseWidth / StartFrame of TestPulseToBaz.cu:119-134, :204-219, :285-300."""
    return fields(field(abi.BAZ_LABEL, serialize=abi.BAZ_TRUNCATE, bits=2),
                  field(abi.BAZ_PULSE_WIDTH, serialize=width_ser, bits=7, ovbytes=ovbytes),
                  field(abi.BAZ_START_FRAME, abi.BAZ_DELTA, serialize=width_ser, bits=7, ovbytes=ovbytes))


def kat_pulses(signals=False):
    """The eight pulses of TestPulseToBaz.cu:140-165 (and :402-436 for the
    signals); MidSignal and SignalM2 read NaN below width 3 (TestingPulse.h:75-92)."""
    import oracle
    p = np.zeros(8, oracle.BAZ_PULSE_DT)
    p["label"] = [A, Cc, G, T, A, Cc, G, T]
    p["width"] = [4, 120, 55, 32, 182, 5, 1, 300]
    gaps = [14, 130, 5, 18, 22, 500, 64, 33]
    start, prev_w = 0, 0
    for i in range(8):
        start += prev_w + gaps[i]
        p["start"][i] = start
        prev_w = int(p["width"][i])
    p["is_base"] = 1
    if signals:
        nan, inf = np.nan, np.inf
        p["pkmax"] = [0, 423.2, 223.645, 623.24, nan, 2123.12, 3613.36, inf]
        p["pkmean"] = [423.2, 223.645, 623.24, nan, 2123.12, 3613.36, inf, 0]
        mid = np.array([223.645, 623.24, nan, 2123.12, 3613.36, inf, 0, 423.2], np.float32)
        m2 = np.array([623.24, nan, 4123.12, 6613.36, inf, 0, 423.2, 223.645], np.float32)
        narrow = p["width"] < 3
        mid[narrow] = nan
        m2[narrow] = nan
        p["pkmid"], p["pkvar"] = mid, m2
    return p


def preset(which):
    from hw_b200 import native
    f = np.zeros(16, abi.BAZ_FIELD_DT)
    n, skip = C.c_uint32(), C.c_int32()
    native.check(native.lib().hw_baz_preset(which, abi.ptr(f), C.byref(n), C.byref(skip)))
    return f[:n.value].copy(), bool(skip.value)


# ---- serializers: TestFieldSerializers.cpp ---------------------------------

# (value, bits, signed, expected) of BazFieldSerializers.Truncate (:36-80)
TRUNCATE = [(0, 1, 0, 0), (1, 1, 0, 1), (2, 1, 0, 0), (3, 1, 0, 1), (3, 3, 0, 3), (5, 3, 0, 5), (7, 3, 0, 7),
            (9, 3, 0, 1), (1 << 33, 32, 0, 0), (1 << 33, 34, 0, 1 << 33),
            (0, 2, 1, 0), (1, 2, 1, 1), (2, 2, 1, -2), (3, 2, 1, -1), (3, 4, 1, 3), (5, 4, 1, 5), (7, 4, 1, 7),
            (9, 4, 1, -7), (1 << 33, 33, 1, 0), (1 << 33, 35, 1, 1 << 33),
            (-1, 2, 1, -1), (-2, 2, 1, -2), (-3, 2, 1, 1), (-3, 4, 1, -3), (-5, 4, 1, -5), (-7, 4, 1, -7),
            (-9, 4, 1, 7), (-(1 << 33), 33, 1, 0), (-(1 << 33), 35, 1, -(1 << 33))]

# (value, bits, overflow bytes, signed) of BazFieldSerializers.SimpleOverflow (:82-140): lossless
SIMPLE = [(0, 1, 1, 0), (1, 1, 1, 0), (2, 1, 1, 0), (3, 1, 1, 0), (3, 3, 1, 0), (5, 3, 1, 0), (7, 3, 1, 0),
          (9, 3, 1, 0), (1 << 33, 32, 8, 0), (1 << 33, 34, 8, 0),
          (0, 2, 1, 1), (1, 2, 1, 1), (2, 2, 1, 1), (3, 2, 1, 1), (3, 4, 1, 1), (5, 4, 1, 1), (7, 4, 1, 1),
          (9, 4, 1, 1), (1 << 33, 33, 8, 1), (1 << 33, 35, 8, 1),
          (-1, 2, 1, 1), (-1, 3, 1, 1), (-2, 2, 1, 1), (-3, 2, 1, 1), (-3, 4, 1, 1), (-5, 4, 1, 1), (-7, 4, 1, 1),
          (-9, 4, 1, 1), (-(1 << 33), 33, 8, 1), (-(1 << 33), 35, 8, 1)]

# (value, bits, signed) of BazFieldSerializers.CompactOverflow (:142-202): lossless, unmasked
COMPACT = [(0, 2, 0), (1, 2, 0), (2, 2, 0), (3, 2, 0), (3, 4, 0), (5, 4, 0), (7, 4, 0), (9, 4, 0),
           (1 << 33, 33, 0), (1 << 33, 35, 0),
           (0, 3, 1), (1, 3, 1), (2, 3, 1), (3, 3, 1), (3, 5, 1), (5, 5, 1), (7, 5, 1), (9, 5, 1),
           (1 << 33, 34, 1), (1 << 33, 36, 1),
           (-1, 3, 1), (-2, 3, 1), (-3, 3, 1), (-3, 5, 1), (-5, 5, 1), (-7, 5, 1), (-9, 5, 1),
           (-(1 << 33), 34, 1), (-(1 << 33), 36, 1)]


def test_oracle_serializers_reproduce_reference_known_answers():
    import oracle
    rt = oracle.baz_serializer_roundtrip
    for v, bits, sgn, want in TRUNCATE:
        got, ov = rt(abi.BAZ_TRUNCATE, bits, 0, sgn, v)
        assert (s64(got) if sgn else got) == want and ov == 0, (v, bits, sgn)
    for v, bits, nb, sgn in SIMPLE:
        got, _ = rt(abi.BAZ_SIMPLE_OVERFLOW, bits, nb, sgn, v)
        assert (s64(got) if sgn else got) == v, (v, bits, nb, sgn)
    # too few overflow bytes truncate (:133-135)
    assert rt(abi.BAZ_SIMPLE_OVERFLOW, 30, 4, 1, -(1 << 33))[0] == 0
    for v, bits, sgn in COMPACT:
        got, _ = rt(abi.BAZ_COMPACT_OVERFLOW, bits, 0, sgn, v, mask=False)
        assert (s64(got) if sgn else got) == v, (v, bits, sgn)
    # overflow byte counts (:137-140, :195-201)
    assert rt(abi.BAZ_SIMPLE_OVERFLOW, 4, 1, 1, 1 << 2)[1] == 0
    assert rt(abi.BAZ_SIMPLE_OVERFLOW, 4, 1, 1, 1 << 5)[1] == 1
    assert rt(abi.BAZ_SIMPLE_OVERFLOW, 4, 4, 1, 1 << 5)[1] == 4
    assert rt(abi.BAZ_SIMPLE_OVERFLOW, 7, 4, 1, 1 << 5)[1] == 0
    assert rt(abi.BAZ_SIMPLE_OVERFLOW, 7, 4, 1, 1 << 9)[1] == 4
    assert rt(abi.BAZ_COMPACT_OVERFLOW, 4, 0, 0, 1 << 2)[1] == 0
    assert rt(abi.BAZ_COMPACT_OVERFLOW, 4, 0, 1, 1 << 2)[1] == 1
    assert rt(abi.BAZ_COMPACT_OVERFLOW, 4, 0, 0, 1 << 5)[1] == 1
    assert rt(abi.BAZ_COMPACT_OVERFLOW, 7, 0, 0, 1 << 5)[1] == 0
    assert rt(abi.BAZ_COMPACT_OVERFLOW, 7, 0, 1, 1 << 9)[1] == 1


# ---- transforms: TestFieldTransforms.cpp ------------------------------------

def _ulps(a, b):
    """Distance in units of the last place (gtest's EXPECT_FLOAT_EQ allows 4)."""
    def key(x):
        i = int(np.float32(x).view(np.int32))
        return i if i >= 0 else -(i & 0x7fffffff)
    return abs(key(a) - key(b))


def test_oracle_float_fixed_codec_reproduces_reference_known_answers():
    """BazTransform.FloatFixedCodec (TestFieldTransforms.cpp:69-186)."""
    import oracle
    rt = lambda v, s, sc, nb: oracle.baz_float_fixed_roundtrip(np.float32(v), s, sc, nb)[0]
    for sgn, v in ((0, 3.125412), (1, -3.125412)):
        for sc, want in ((10, 3.1), (100, 3.13), (1000, 3.125), (30, 3.13333333)):
            assert _ulps(rt(v, sgn, sc, 2), np.float32(want if sgn == 0 else -want)) <= 4, (v, sc)
    inf = np.float32(np.inf)
    for sgn in (0, 1):
        for sc in (10, 100):
            for nb in (1, 4, 8):
                assert np.isnan(rt(np.nan, sgn, sc, nb))
                assert rt(inf, sgn, sc, nb) == inf
                assert rt(-inf, sgn, sc, nb) == -inf
    big = np.float32(np.finfo(np.float32).max) - np.float32(1000)
    assert rt(big, 0, 2, 8) == inf and _ulps(rt(big, 0, 1, 8), big) <= 4
    assert rt(big, 1, 2, 8) == inf and _ulps(rt(big, 1, 1, 8), big) <= 4
    low = np.float32(np.finfo(np.float32).min) + np.float32(1000)
    assert rt(low, 0, 2, 8) == -inf and _ulps(rt(low, 0, 1, 8), -inf) <= 4
    assert rt(low, 1, 2, 8) == -inf and _ulps(rt(low, 1, 1, 8), low) <= 4
    for sgn in (0, 1):
        for code in (0, 1, 2):                       # the special codes as inputs
            assert rt(code, sgn, 1, 1) == code
    for v in (256, 255, 254, 253):
        assert rt(v, 0, 1, 1) == inf
    assert rt(252, 0, 1, 1) == 252
    for v in (252, 127, 126, 125):
        assert rt(v, 1, 1, 1) == inf
    assert rt(124, 1, 1, 1) == 124
    assert rt(-127, 1, 1, 1) == -inf and rt(-124, 1, 1, 1) == -124
    assert rt(7623.531, 0, 10, 2) == inf and abs(rt(7623.531, 0, 10, 3) - 7623.5) < 1e-2
    assert rt(3623.531, 1, 10, 2) == inf and abs(rt(3623.531, 1, 10, 3) - 3623.5) < 1e-2
    assert rt(-3623.531, 1, 10, 2) == -inf and abs(rt(-3623.531, 1, 10, 3) + 3623.5) < 1e-2


def test_oracle_delta_transform_reproduces_reference_known_answers():
    """BazTransform.DeltaCompression (TestFieldTransforms.cpp:295-322) through a
    16-bit truncated start-frame field: the main bytes are the deltas."""
    import oracle
    for sgn, starts, deltas in ((0, [10, 20, 30, 50, 55], [10, 10, 10, 20, 5]),
                                (1, [10, 20, 10, 15, 5], [10, 10, -10, 5, -10])):
        f = fields(field(abi.BAZ_START_FRAME, abi.BAZ_DELTA, abi.BAZ_TRUNCATE, bits=16, signed=bool(sgn)))
        p = np.zeros(len(starts), oracle.BAZ_PULSE_DT)
        p["start"] = starts
        data = oracle.baz_encode_values(f, p)
        assert data.view(np.int16 if sgn else np.uint16).tolist() == deltas
        back, used = oracle.baz_decode_values(f, data, len(starts))
        assert used == len(data) and back["start"].tolist() == starts


# ---- whole pulses: TestPulseToBaz.cu, TestBazRoundTrip.cpp ------------------

def test_oracle_kestrel_lossy_truncate():
    """PulseToBaz.KestrelLossyTruncate (TestPulseToBaz.cu:115-196): 16 bytes,
    widths and start deltas modulo 128."""
    import oracle
    f = kestrel(abi.BAZ_TRUNCATE)
    p = kat_pulses()
    data = oracle.baz_encode_values(f, p)
    assert len(data) == 16
    back, used = oracle.baz_decode_values(f, data, 8)
    assert used == 16
    assert back["label"].tolist() == p["label"].tolist()
    assert (back["width"] == p["width"] % 128).all()
    d_in = np.diff(np.concatenate([[0], p["start"].astype(np.int64)]))
    d_out = np.diff(np.concatenate([[0], back["start"].astype(np.int64)]))
    assert (d_out == d_in % 128).all()


@pytest.mark.parametrize("ser,ovbytes,length", [(abi.BAZ_SIMPLE_OVERFLOW, 4, 32), (abi.BAZ_COMPACT_OVERFLOW, 0, 24)])
def test_oracle_kestrel_lossless(ser, ovbytes, length):
    """PulseToBaz.KestrelLosslessSimple (:200-273) and KestrelLosslessCompact
    (:277-350), BazRoundTrip (TestBazRoundTrip.cpp:41-170): 32 and 24 bytes,
    every field back."""
    import oracle
    f = kestrel(ser, ovbytes)
    p = kat_pulses()
    data = oracle.baz_encode_values(f, p)
    assert len(data) == length
    back, used = oracle.baz_decode_values(f, data, 8)
    assert used == length
    for k in ("label", "width", "start"):
        assert back[k].tolist() == p[k].tolist(), k


def test_presets_are_the_basecaller_encodings():
    """PulseGroups.h:42-94; the production encoding is KestrelLosslessCompact,
    PulseToBaz.Params (TestPulseToBaz.cu:516-586)."""
    prod, skip = preset(abi.BAZ_PRODUCTION)
    assert skip and prod.tobytes() == kestrel(abi.BAZ_COMPACT_OVERFLOW).tobytes()
    internal, skip = preset(abi.BAZ_INTERNAL)
    assert not skip and internal[:3].tobytes() == prod.tobytes()
    names = internal["name"].tolist()
    assert names[3:] == [abi.BAZ_PKMAX, abi.BAZ_PKMID, abi.BAZ_PKMEAN, abi.BAZ_PKVAR, abi.BAZ_IS_BASE]
    for f in internal[3:7]:
        assert f["transform"] == abi.BAZ_FLOAT_FIXED and f["scale"] == 10 and f["transform_bytes"] == 2
        assert f["serialize"] == abi.BAZ_SIMPLE_OVERFLOW and f["overflow_bytes"] == 2
    assert internal["num_bits"][3:].tolist() == [8, 8, 8, 7, 1]
    assert internal["store_signed"][3:].tolist() == [1, 1, 1, 0, 0]


def test_oracle_internal_mode():
    """PulseToBaz.InternalMode (TestPulseToBaz.cu:352-513) and
    BazRoundTrip.InternalMode (TestBazRoundTrip.cpp:172-330): 86 bytes; each
    signal within 1/scale, or non-finite above the code's range."""
    import oracle
    f, _ = preset(abi.BAZ_INTERNAL)
    p = kat_pulses(signals=True)
    data = oracle.baz_encode_values(f, p)
    assert len(data) == 86
    back, used = oracle.baz_decode_values(f, data, 8)
    assert used == 86
    for k in ("label", "width", "start"):
        assert back[k].tolist() == p[k].tolist(), k
    for k, sgn in (("pkmax", 1), ("pkmean", 1), ("pkmid", 1), ("pkvar", 0)):
        mx = np.float32(32767 if sgn else 65535) / np.float32(10)
        for i in range(8):
            t, c = p[k][i], back[k][i]
            if np.isnan(t):
                assert np.isnan(c), (k, i)
            elif t < mx:
                assert abs(t - c) <= 0.1 + 1e-6, (k, i)
            else:
                assert not np.isfinite(c), (k, i)


def test_oracle_nominal_sizes():
    """Groups (ObjectToBaz.h:373-393): 2 bytes a production pulse, 6 an
    internal one (Label/Width/Start, then Pkmax, Pkmid, Pkmean alone, then
    Pkvar with IsBase) when nothing overflows."""
    import oracle
    p = np.zeros(1, oracle.BAZ_PULSE_DT)
    p["width"], p["start"], p["pkmax"], p["pkmid"], p["pkmean"], p["pkvar"] = 3, 5, 1.0, 1.0, 1.0, 1.0
    assert len(oracle.baz_encode_values(preset(abi.BAZ_PRODUCTION)[0], p)) == 2
    assert len(oracle.baz_encode_values(preset(abi.BAZ_INTERNAL)[0], p)) == 6


def _baz_values(hp):
    """PulseFieldAccessors.h:43-68 on numpy hw_pulse records."""
    import oracle
    b = np.zeros(len(hp), oracle.BAZ_PULSE_DT)
    b["label"], b["start"], b["width"] = hp["label"], hp["start"], hp["width"]
    b["is_base"] = (hp["is_reject"] == 0).astype(np.uint8)
    tenth = np.float32(0.1)
    narrow = hp["width"] < 3
    b["pkmax"] = hp["max_signal"].astype(np.float32) * tenth
    b["pkmean"] = hp["mean_signal"].astype(np.float32) * tenth
    b["pkmid"] = np.where(narrow, np.float32(np.nan), hp["mid_signal"].astype(np.float32) * tenth)
    b["pkvar"] = np.where(narrow, np.float32(np.nan), hp["signal_m2"])
    return b


def random_pulses(rng, num_zmw, cap, max_len=None):
    """Basecaller pulses with every kind of value the encodings meet: long
    widths and gaps (compact overflow of 1 to 3 bytes), rejects, widths
    below 3, signals above the fixed-point range, NaN, infinite and negative
    SignalM2."""
    p = np.zeros((num_zmw, cap), abi.PULSE_DT)
    lens = rng.integers(0, (cap if max_len is None else max_len) + 1, num_zmw).astype(np.uint32)
    w = rng.choice([1, 2, 3, 5, 60, 200, 20000], size=(num_zmw, cap), p=[.1, .1, .3, .3, .1, .07, .03])
    gap = rng.choice([0, 3, 100, 5000, 300000], size=(num_zmw, cap), p=[.2, .4, .25, .1, .05])
    start = rng.integers(0, 1 << 20, num_zmw)[:, None] + np.cumsum(w + gap, axis=1) - w
    p["start"] = start.astype(np.uint32)
    p["width"] = w
    p["max_signal"] = rng.choice([0, 50, 4232, 32760, 32770, 65535], size=(num_zmw, cap))
    p["mean_signal"] = rng.integers(0, 65536, (num_zmw, cap))
    p["mid_signal"] = rng.integers(0, 40000, (num_zmw, cap))
    m2 = rng.choice([0.0, 1.5, 6553.2, 6553.6, 1e7, np.inf, np.nan, -5.0], size=(num_zmw, cap))
    p["signal_m2"] = m2.astype(np.float32)
    p["label"] = rng.integers(0, 4, (num_zmw, cap))
    p["is_reject"] = rng.random((num_zmw, cap)) < 0.15
    return p, lens


@pytest.mark.parametrize("which", [abi.BAZ_PRODUCTION, abi.BAZ_INTERNAL])
def test_oracle_chunk_equals_per_zmw_encoding(which):
    """The chunk entry (PrelimHQFilter append) equals each ZMW's pulses encoded
    alone, rejects left out in production; the delta state carries over."""
    import oracle
    f, skip = preset(which)
    rng = np.random.default_rng(3)
    nz, cap = 40, 24
    enc = oracle.BazEncoder(f, skip, nz)
    last = np.zeros((nz, len(f)), np.uint64)
    for chunk in range(3):
        p, lens = random_pulses(rng, nz, cap)
        data, off = enc(p, lens, cap)
        for z in range(nz):
            hp = p[z, :lens[z]]
            if skip:
                hp = hp[hp["is_reject"] == 0]
            want = oracle.baz_encode_values(f, _baz_values(hp), last[z])
            assert data[off[z]:off[z + 1]].tobytes() == want.tobytes(), (chunk, z)


def test_oracle_zmw_stride_leaves_other_zmws_empty():
    """zmwOutputStride (PrelimHQFilter.cpp:107-118): ZMW 0, 4, 8 ... of each
    lane encoded, the others empty."""
    import oracle
    f, skip = preset(abi.BAZ_PRODUCTION)
    rng = np.random.default_rng(5)
    p, lens = random_pulses(rng, 256, 16)
    lens[:] = np.maximum(lens, 1)
    every = oracle.BazEncoder(f, skip, 256)(p, lens, 16)
    data, off = oracle.BazEncoder(f, skip, 256, zmw_stride=4)(p, lens, 16)
    for z in range(256):
        got = data[off[z]:off[z + 1]].tobytes()
        want = every[0][every[1][z]:every[1][z + 1]].tobytes() if z % 4 == 0 else b""
        assert got == want, z


def test_encoder_rejects_bad_field_lists():
    """Checked before any device work: no GPU needed."""
    from hw_b200 import native
    lib = native.lib()
    h = C.c_void_p()
    bad = [field(abi.BAZ_PKMAX, abi.BAZ_NOOP, bits=8),                          # a signal needs the codec
           field(abi.BAZ_LABEL, abi.BAZ_FLOAT_FIXED, scale=10, tbytes=2),        # an integer field does not
           field(abi.BAZ_LABEL, bits=0), field(abi.BAZ_LABEL, bits=31),
           field(abi.BAZ_PKVAR, abi.BAZ_FLOAT_FIXED, scale=10, tbytes=8),
           field(abi.BAZ_START_FRAME, abi.BAZ_DELTA, abi.BAZ_COMPACT_OVERFLOW, bits=15, signed=True),
           field(abi.BAZ_PULSE_WIDTH, serialize=abi.BAZ_SIMPLE_OVERFLOW, ovbytes=0)]
    for b in bad:
        f = fields(b)
        assert lib.hw_baz_encoder_create(abi.ptr(f), 1, 0, 64, C.byref(h)) == 1
    f = fields(*[field(abi.BAZ_LABEL, bits=2)] * 17)
    assert lib.hw_baz_encoder_create(abi.ptr(f), 17, 0, 64, C.byref(h)) == 1
    f = fields(field(abi.BAZ_LABEL, bits=2))
    assert lib.hw_baz_encoder_create(abi.ptr(f), 1, 0, 0, C.byref(h)) == 1


# ---- the CUDA encoder --------------------------------------------------------

CUSTOM = [
    # every serializer and transform, signed fields, 1- and 3-byte codes, a
    # group closed by the 64-bit limit
    lambda: fields(field(abi.BAZ_START_FRAME, abi.BAZ_DELTA, abi.BAZ_SIMPLE_OVERFLOW, bits=12, ovbytes=4),
                   field(abi.BAZ_PULSE_WIDTH, abi.BAZ_NOOP, abi.BAZ_COMPACT_OVERFLOW, bits=5),
                   field(abi.BAZ_PKMEAN, abi.BAZ_FLOAT_FIXED, abi.BAZ_SIMPLE_OVERFLOW, bits=9, signed=True,
                         scale=3, tbytes=3, ovbytes=3),
                   field(abi.BAZ_PKVAR, abi.BAZ_FLOAT_FIXED, abi.BAZ_COMPACT_OVERFLOW, bits=6, scale=100,
                         tbytes=1),
                   field(abi.BAZ_LABEL, serialize=abi.BAZ_TRUNCATE, bits=3, signed=True),
                   field(abi.BAZ_START_FRAME, abi.BAZ_DELTA, abi.BAZ_COMPACT_OVERFLOW, bits=13, signed=True),
                   field(abi.BAZ_PKMAX, abi.BAZ_FLOAT_FIXED, abi.BAZ_TRUNCATE, bits=30, signed=True, scale=7,
                         tbytes=7),
                   field(abi.BAZ_IS_BASE, bits=1)),
]


def _gpu_vs_oracle(f, skip, chunks, nz, cap, seed, max_len=None, stride=1):
    import torch
    import oracle
    from hw_b200 import filters as Fl
    rng = np.random.default_rng(seed)
    gpu = Fl.BazEncoder(nz, fields=f, skip_rejects=skip, zmw_stride=stride)
    ref = oracle.BazEncoder(f, skip, nz, zmw_stride=stride)
    total = 0
    for _ in range(chunks):
        p, lens = random_pulses(rng, nz, cap, max_len)
        want, woff = ref(p, lens, cap)
        d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
        d_l = torch.from_numpy(lens.view(np.int32)).cuda()
        got, goff = gpu(d_p, d_l, cap)
        assert goff.cpu().numpy().astype(np.uint64).tolist() == woff.tolist()
        assert got.cpu().numpy().tobytes() == want.tobytes()
        kept = np.minimum(lens, cap)[:, None] > np.arange(cap)[None, :]
        if skip:
            kept &= p["is_reject"] == 0
        kept[(np.arange(nz) % 64) % stride != 0] = False
        assert (gpu.events.cpu().numpy() == kept.sum(axis=1)).all()
        total += len(want)
    gpu.close()
    return total


@pytest.mark.gpu
@pytest.mark.parametrize("which", [abi.BAZ_PRODUCTION, abi.BAZ_INTERNAL])
def test_gpu_encoder_matches_oracle_on_presets(which):
    """160 tiles of 128 ZMWs: the look-back crosses several 32-tile windows."""
    f, skip = preset(which)
    assert _gpu_vs_oracle(f, skip, chunks=3, nz=20400, cap=24, seed=11) > 0


@pytest.mark.gpu
@pytest.mark.parametrize("make", CUSTOM)
@pytest.mark.parametrize("skip", [False, True])
def test_gpu_encoder_matches_oracle_on_custom_fields(make, skip):
    assert _gpu_vs_oracle(make(), skip, chunks=3, nz=700, cap=32, seed=5) > 0


@pytest.mark.gpu
def test_gpu_encoder_edges():
    """Empty chunks, a single ZMW, ZMW counts off the tile size, and a too
    small buffer (HW_ERR_OUT_OF_MEMORY with the offsets set, state unchanged)."""
    import torch
    import oracle
    from hw_b200 import filters as Fl, native
    f, skip = preset(abi.BAZ_PRODUCTION)
    assert _gpu_vs_oracle(f, skip, chunks=2, nz=1, cap=8, seed=1) >= 0
    assert _gpu_vs_oracle(f, skip, chunks=2, nz=129, cap=8, seed=2) >= 0
    assert _gpu_vs_oracle(f, skip, chunks=2, nz=77, cap=16, seed=3, max_len=0) == 0
    # too small: nothing written, the delta state unchanged
    nz, cap = 100, 16
    rng = np.random.default_rng(9)
    p, lens = random_pulses(rng, nz, cap)
    lens[:] = np.maximum(lens, 1)
    gpu = Fl.BazEncoder(nz, fields=f, skip_rejects=False)
    ref = oracle.BazEncoder(f, False, nz)
    d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
    d_l = torch.from_numpy(lens.view(np.int32)).cuda()
    small = torch.zeros(4, dtype=torch.uint8, device="cuda")
    total = C.c_uint64()
    rc = native.lib().hw_baz_encode(gpu._h, C.c_void_p(d_p.data_ptr()), C.c_void_p(d_l.data_ptr()), cap,
                                    C.c_void_p(small.data_ptr()), 4, C.c_void_p(gpu.offsets.data_ptr()), None,
                                    C.byref(total), None)
    assert rc == abi.HW_ERR_OUT_OF_MEMORY and total.value > 4
    want, woff = ref(p, lens, cap)
    assert gpu.offsets.cpu().numpy().astype(np.uint64).tolist() == woff.tolist()
    # a buffer of exactly the chunk's bytes; then the next chunk: the state
    # was left as it was by the refused call
    exact = torch.zeros(total.value, dtype=torch.uint8, device="cuda")
    rc = native.lib().hw_baz_encode(gpu._h, C.c_void_p(d_p.data_ptr()), C.c_void_p(d_l.data_ptr()), cap,
                                    C.c_void_p(exact.data_ptr()), total.value, C.c_void_p(gpu.offsets.data_ptr()),
                                    None, C.byref(total), None)
    assert rc == 0 and exact.cpu().numpy().tobytes() == want.tobytes()
    want, _ = ref(p, lens, cap)
    got, _ = gpu(d_p, d_l, cap)
    assert got.cpu().numpy().tobytes() == want.tobytes()


@pytest.mark.gpu
def test_gpu_encoder_zmw_stride():
    f, skip = preset(abi.BAZ_PRODUCTION)
    assert _gpu_vs_oracle(f, skip, chunks=3, nz=1000, cap=24, seed=13, stride=4) > 0


@pytest.mark.gpu
def test_gpu_encoder_production_fields_keeping_rejects():
    """The production fields with rejected pulses kept: the general field
    path of the kernel (the constant production path skips rejects)."""
    f, _ = preset(abi.BAZ_PRODUCTION)
    assert _gpu_vs_oracle(f, False, chunks=3, nz=900, cap=40, seed=8) > 0
    f, _ = preset(abi.BAZ_INTERNAL)
    assert _gpu_vs_oracle(f, True, chunks=3, nz=900, cap=40, seed=9) > 0


@pytest.mark.gpu
def test_gpu_encoder_on_chain_pulses_round_trip():
    """Pulses of the CUDA chain encoded on the GPU equal the oracle's bytes, and
    decode back to the pulses' labels, widths and starts."""
    import torch
    import oracle
    import synth
    from hw_b200 import filters as Fl, workloads
    cfg = workloads.small_config()
    lanes, Fc, chunks = 3, 512, 8
    nz = lanes * abi.LANE
    tr = synth.traces(lanes, Fc * chunks, seed=4)
    an = Fl.BatchAnalyzer(cfg, 0, lanes, Fc)
    cap = cfg.max_calls_per_zmw
    f, skip = preset(abi.BAZ_PRODUCTION)
    gpu = Fl.BazEncoder(nz, fields=f, skip_rejects=skip)
    ref = oracle.BazEncoder(f, skip, nz)
    last = np.zeros((nz, len(f)), np.uint64)
    decoded = 0
    for c in range(chunks):
        chunk = torch.from_numpy(np.ascontiguousarray(tr[:, c * Fc:(c + 1) * Fc])).cuda()
        pulses, lens, ovf, em, est = an(chunk, c * Fc)
        if not em:
            continue
        got, goff = gpu(pulses, lens, cap)
        hp = Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(nz, cap)
        hl = lens.cpu().numpy().astype(np.uint32).reshape(nz)
        want, woff = ref(hp, hl, cap)
        assert got.cpu().numpy().tobytes() == want.tobytes()
        goff = goff.cpu().numpy().astype(np.uint64)
        for z in range(nz):
            kept = hp[z, :hl[z]]
            kept = kept[kept["is_reject"] == 0]
            back, used = oracle.baz_decode_values(f, want[goff[z]:goff[z + 1]], len(kept), last[z])
            assert used == goff[z + 1] - goff[z]
            for k in ("label", "width", "start"):
                assert back[k].tolist() == kept[k].tolist()
            decoded += len(kept)
    assert decoded > 1000


@pytest.mark.gpu
def test_gpu_encoder_async_calls_in_a_row():
    """Encodings enqueued back to back: each continues the state of the last
    one that fit; a call whose buffer is too small leaves the state, and the
    result call reports the last one."""
    import torch
    import oracle
    from hw_b200 import filters as Fl
    f, skip = preset(abi.BAZ_PRODUCTION)
    nz, cap = 3000, 24
    rng = np.random.default_rng(21)
    chunks = [random_pulses(rng, nz, cap) for _ in range(4)]
    ref = oracle.BazEncoder(f, skip, nz)
    want = [ref(*chunks[0], cap)[0], None, ref(*chunks[2], cap)[0], ref(*chunks[3], cap)[0]]
    gpu = Fl.BazEncoder(nz, fields=f, skip_rejects=skip)
    outs, offs, keep = [], [], []
    for c, (p, lens) in enumerate(chunks):
        d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
        d_l = torch.from_numpy(lens.view(np.int32)).cuda()
        size = 8 if c == 1 else len(want[c]) + 64
        outs.append(torch.zeros(size, dtype=torch.uint8, device="cuda"))
        offs.append(torch.zeros(nz + 1, dtype=torch.int64, device="cuda"))
        keep.append((d_p, d_l))
        gpu.enqueue(d_p, d_l, cap, outs[-1], offs[-1])
    torch.cuda.synchronize()
    assert gpu.result() == len(want[3])
    for c in (0, 2, 3):
        n = int(offs[c][-1].item())
        assert n == len(want[c])
        assert outs[c][:n].cpu().numpy().tobytes() == want[c].tobytes(), c


@pytest.mark.gpu
def test_gpu_encoder_chip_size_properties():
    """1,048,576 ZMWs (8192 tiles): offsets rise by each ZMW's bytes, event
    counts equal the kept pulses, and a sample of ZMWs spread over the whole
    chip decodes back to their pulses' labels, widths and starts (delta state
    from the previous chunk carried)."""
    import torch
    import oracle
    from hw_b200 import filters as Fl
    nz, cap = 1 << 20, 12
    f, skip = preset(abi.BAZ_PRODUCTION)
    rng = np.random.default_rng(17)
    gpu = Fl.BazEncoder(nz, fields=f, skip_rejects=skip)
    sample = np.sort(rng.choice(nz, 512, replace=False))
    last = np.zeros((nz, len(f)), np.uint64)
    for chunk in range(2):
        p, lens = random_pulses(rng, nz, cap)
        d_p = torch.from_numpy(p.view(np.uint8).reshape(-1)).cuda()
        d_l = torch.from_numpy(lens.view(np.int32)).cuda()
        data, off = gpu(d_p, d_l, cap)
        off = off.cpu().numpy().astype(np.uint64)
        data = data.cpu().numpy()
        kept = (np.minimum(lens, cap)[:, None] > np.arange(cap)[None, :]) & (p["is_reject"] == 0)
        n_kept = kept.sum(axis=1)
        assert (gpu.events.cpu().numpy() == n_kept).all()
        assert off[0] == 0 and (np.diff(off.astype(np.int64)) >= 0).all() and off[-1] == len(data)
        for z in sample:
            k = p[z, :lens[z]]
            k = k[k["is_reject"] == 0]
            back, used = oracle.baz_decode_values(f, data[off[z]:off[z + 1]], len(k), last[z])
            assert used == off[z + 1] - off[z]
            for name in ("label", "width", "start"):
                assert back[name].tolist() == k[name].tolist(), (chunk, z, name)


@pytest.mark.gpu
def test_gpu_encoder_bounded_wait_reports_timeout():
    """A tile that never publishes its count (a test hook): the tiles after
    it stop waiting after the poll bound, the call returns HW_ERR_TIMEOUT
    with the delta state unchanged, and the next call encodes the chunk as
    the oracle does -- the context stays usable, nothing faults or hangs."""
    import torch
    import oracle
    from hw_b200 import filters as Fl, native
    f, skip = preset(abi.BAZ_PRODUCTION)
    nz, cap = 128 * 40, 16
    rng = np.random.default_rng(31)
    p, lens = random_pulses(rng, nz, cap)
    gpu = Fl.BazEncoder(nz, fields=f, skip_rejects=skip)
    ref = oracle.BazEncoder(f, skip, nz)
    d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
    d_l = torch.from_numpy(lens.view(np.int32)).cuda()
    lib = native.lib()
    assert lib.hw_baz_encoder_set_wait_limit(gpu._h, 4096, 5) == 0
    with pytest.raises(native.HwError) as err:
        gpu(d_p, d_l, cap)
    assert err.value.code == 7 and "HW_ERR_TIMEOUT" in str(err.value)
    assert lib.hw_baz_encoder_set_wait_limit(gpu._h, 1 << 22, -1) == 0
    want, woff = ref(p, lens, cap)
    got, goff = gpu(d_p, d_l, cap)
    assert goff.cpu().numpy().astype(np.uint64).tolist() == woff.tolist()
    assert got.cpu().numpy().tobytes() == want.tobytes()
