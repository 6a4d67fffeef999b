"""The multi-rank path on the CPU: two `gloo` ranks, one process each.

Each rank analyses its own share of the lanes through the chain (oracle
backend, since this host has no GPU) with no data exchange; rank 0 gathers
the pulses of both ranks and checks them against one process analysing all
lanes, and every rank checks the timing max-reduction.  This is the
structure `bench.py --gpus N` uses with NCCL, one GPU per rank.
"""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LANES, F, CHUNKS = 3, 512, 8


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _run_pool(lanes_slice, tr, cfg):
    import harness
    lanes = lanes_slice[1] - lanes_slice[0]
    pipe = harness.Pipeline(harness.OracleBackend(cfg, lanes, F), cfg)
    out = []
    for c in range(CHUNKS):
        chunk = np.ascontiguousarray(tr[lanes_slice[0]:lanes_slice[1], c * F:(c + 1) * F])
        r = pipe.process(chunk, c * F)
        if "pulses" in r:
            p, lens, ovf, _ = r["pulses"]
            out.append((c, p.view(np.uint8).copy(), lens.copy(), ovf.copy()))
    return out


def _worker(rank, world, port, q):
    try:
        for p in (ROOT, os.path.join(ROOT, "tests"), os.path.join(ROOT, "oracle")):
            sys.path.insert(0, p)
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        import synth
        from hw_b200 import shard, workloads
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
        cfg = workloads.small_config()
        tr = synth.traces(LANES, F * CHUNKS, seed=13)
        start, count = shard.lane_range(rank, world, LANES)
        mine = _run_pool((start, start + count), tr, cfg)
        # gather every rank's pulse records (object collective over gloo)
        gathered = [None] * world
        dist.all_gather_object(gathered, (start, count, mine))
        t = shard.max_over_ranks(10.0 * (rank + 1))
        dist.barrier()
        dist.destroy_process_group()
        if rank == 0:
            full = _run_pool((0, LANES), tr, cfg)
            assert sum(c for _, c, _ in gathered) == LANES
            assert [s for s, _, _ in gathered] == [0, gathered[0][1]]
            for ci, (c, p, lens, ovf) in enumerate(full):
                lanes_p = p.reshape(LANES, -1)
                for s, n, recs in gathered:
                    c2, p2, l2, o2 = recs[ci]
                    assert c2 == c
                    assert np.array_equal(lanes_p[s:s + n].ravel(), p2.ravel())
                    assert np.array_equal(lens[s:s + n], l2) and np.array_equal(ovf[s:s + n], o2)
            assert len(full) > 0
        q.put((rank, "ok", t))
    except BaseException as e:      # report to the parent instead of hanging it
        import traceback
        q.put((rank, "".join(traceback.format_exception(e)), None))


def test_two_gloo_ranks_shard_lanes_without_exchange():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = {}
    try:
        for _ in range(2):
            rank, status, t = q.get(timeout=300)
            results[rank] = (status, t)
    finally:
        for p in procs:
            p.join(timeout=30)
            if p.is_alive():
                p.kill()
    for rank in (0, 1):
        status, t = results[rank]
        assert status == "ok", f"rank {rank}:\n{status}"
        assert t == 20.0


@pytest.mark.parametrize("world", [1, 2, 3, 4, 8])
def test_lane_range_partitions(world):
    from hw_b200 import shard
    for total in (1, 7, 16384, 16385):
        if total < world:
            continue
        ranges = [shard.lane_range(r, world, total) for r in range(world)]
        assert ranges[0][0] == 0
        for (s0, n0), (s1, _) in zip(ranges, ranges[1:]):
            assert s0 + n0 == s1
        assert sum(n for _, n in ranges) == total
        assert max(n for _, n in ranges) - min(n for _, n in ranges) <= 1


def test_weak_scaling_offsets_are_disjoint():
    from hw_b200 import shard
    z = 1 << 20
    offs = [shard.zmw_offset(r, z) for r in range(8)]
    assert offs == [r * z for r in range(8)]
    with pytest.raises(ValueError):
        shard.lane_range(2, 2, 10)
