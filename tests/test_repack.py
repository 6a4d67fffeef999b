"""Ingest repacking (BlockRepacker): the reference's chunk generator and
validation pattern (appModules/test/TestBlockRepacker.cpp:63-330) restated;
the oracle must place every value at its ZMW and frame, and the CUDA gather
must equal the oracle byte for byte."""
import numpy as np
import pytest

from hw_b200 import abi


def make_chunk(num_zmw, start_frame, num_frames, packet_frames, packet_blocks, block_width, encoding,
               irregular=(0, 0), shuffle_seed=1):
    """GeneratePacketsChunk / GeneratePacket: each value holds the low half of
    its frame number over the low half of its ZMW number."""
    dt = np.int16 if encoding == 0 else np.uint8
    bits = np.dtype(dt).itemsize * 8 // 2
    mask = (1 << bits) - 1
    packets, blobs, off = [], [], 0
    for i in range(num_frames // packet_frames):
        frame0 = start_frame + i * packet_frames
        z, k = 0, 1
        while z < num_zmw:
            nb = irregular[1] if irregular[0] and k % irregular[0] else packet_blocks
            end = min(num_zmw, z + nb * block_width)
            nb = (end - z) // block_width
            zz = z + np.arange(nb * block_width).reshape(nb, 1, block_width)
            ff = frame0 + np.arange(packet_frames).reshape(1, packet_frames, 1)
            vals = (((ff & mask) << bits) | (zz & mask)).astype(np.int64)
            blob = vals.astype(np.uint16 if dt == np.int16 else np.uint8).view(dt)
            packets.append((off, z, frame0, packet_frames, block_width, nb, 0))
            raw = blob.tobytes()
            pad = (-len(raw)) % 16
            blobs.append(raw + b"\0" * pad)
            off += len(raw) + pad
            z = end
            k += 1
    order = np.random.default_rng(shuffle_seed).permutation(len(packets))    # packets arrive in any order
    table = np.array([packets[i] for i in order], abi.SENSOR_PACKET_DT)
    return table, np.frombuffer(b"".join(blobs), np.uint8)


def expected(num_zmw, lanes_per_pool, F, start_frame, encoding):
    dt = np.int16 if encoding == 0 else np.uint8
    bits = np.dtype(dt).itemsize * 8 // 2
    mask = (1 << bits) - 1
    lanes = num_zmw // 64
    out = []
    for p0 in range(0, lanes, lanes_per_pool):
        L = min(lanes_per_pool, lanes - p0)
        zz = (p0 + np.arange(L)).reshape(L, 1, 1) * 64 + np.arange(64).reshape(1, 1, 64)
        ff = start_frame + np.arange(F).reshape(1, F, 1)
        vals = ((ff & mask) << bits) | (zz & mask)
        out.append(vals.astype(np.uint16 if dt == np.int16 else np.uint8).view(dt))
    return out


def oracle_repack(num_zmw, lanes_per_pool, F, encoding, table, data, start_frame):
    import oracle
    dt = np.int16 if encoding == 0 else np.uint8
    lanes = num_zmw // 64
    chunks = [np.zeros((min(lanes_per_pool, lanes - p0), F, 64), dt) for p0 in range(0, lanes, lanes_per_pool)]
    oracle.repack(num_zmw, lanes_per_pool, F, encoding, table, data, start_frame, chunks)
    return chunks


# (NumZmw, BatchBlocks, PacketFrames, PacketBlocks, PacketBlockWidth, encoding): the reference sweep's
# shapes at a CPU-sized chip
CASES = [(4096, 16, 64, 50, 32, 0), (4096, 16, 256, 50, 64, 0), (4096, 8, 64, 50, 128, 0),
         (16384, 256, 256, 50, 128, 0), (4096, 16, 64, 50, 64, 1), (16384, 256, 256, 50, 128, 1)]


@pytest.mark.parametrize("case", CASES)
def test_oracle_places_every_value(case):
    num_zmw, bb, pf, pb, bw, enc = case
    F = 256
    for c in range(3):                       # ThreeChunkRepack
        table, data = make_chunk(num_zmw, c * F, F, pf, pb, bw, enc)
        got = oracle_repack(num_zmw, bb, F, enc, table, data, c * F)
        for g, w in zip(got, expected(num_zmw, bb, F, c * F, enc)):
            assert np.array_equal(g, w)


def test_oracle_irregular_packets():
    num_zmw, F = 8192, 256
    table, data = make_chunk(num_zmw, 0, F, 64, 50, 64, 0, irregular=(3, 7))
    got = oracle_repack(num_zmw, 16, F, 0, table, data, 0)
    for g, w in zip(got, expected(num_zmw, 16, F, 0, 0)):
        assert np.array_equal(g, w)


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_repack_equals_oracle(case):
    import torch
    from hw_b200 import filters as Fl
    num_zmw, bb, pf, pb, bw, enc = case
    F = 256
    rp = Fl.Repacker(num_zmw, bb, F, "int16" if enc == 0 else "uint8")
    chunks = rp.new_chunks()
    for c in range(3):
        table, data = make_chunk(num_zmw, c * F, F, pf, pb, bw, enc, irregular=(4, 9) if c == 1 else (0, 0))
        d = torch.from_numpy(data.copy()).cuda()
        rp(table, d, c * F, chunks)
        torch.cuda.synchronize()
        want = oracle_repack(num_zmw, bb, F, enc, table, data, c * F)
        for g, w in zip(chunks, want):
            assert np.array_equal(g.cpu().numpy(), w)
        for g, w in zip(chunks, expected(num_zmw, bb, F, c * F, enc)):
            assert np.array_equal(g.cpu().numpy(), w)


@pytest.mark.gpu
def test_gpu_repack_rejects_bad_packets():
    import torch
    from hw_b200 import filters as Fl
    from hw_b200.native import HwError
    rp = Fl.Repacker(4096, 16, 256)
    chunks = rp.new_chunks()
    table, data = make_chunk(4096, 0, 256, 64, 50, 64, 0)
    d = torch.from_numpy(data.copy()).cuda()
    bad = table.copy()
    bad["start_frame"][0] = 256                 # outside the chunk
    with pytest.raises(HwError):
        rp(bad, d, 0, chunks)
    bad = table.copy()
    bad["block_width"][0] = 48                  # not a whole number of cache lines
    with pytest.raises(HwError):
        rp(bad, d, 0, chunks)
