#!/usr/bin/env python
"""Throughput of the smrt-basecaller trace-analysis chain on B200.

Workload (chip scale): 1,048,576 ZMWs = 16,384 lanes of 64, as 4 pools of 4096
lanes, 512-frame int16 chunks from the trace generator (lognormal gain sigma
0.2, 15% empty ZMWs, 0.05 DN/frame baseline random walk), reference default
analysis parameters (MultiScaleLarge baseliner, dynamic estimation: every
pool re-estimates its detection models every 4000 frames, staggered by
pool).  The run first streams the start-up chunks (untimed) until every pool
is in its periodic estimation cycle; a step is then one chunk of the whole
chip through baseliner -> statistics -> histogram -> (EM when due) ->
labeler -> pulses (+ HF metrics), each pool through its own hw_chunk_fused
engine, the four engines on four streams (--groups, --streams).  The
8-step estimation cycle runs one EM per pool, so K steps from a given phase
of the cycle hold a phase-dependent number of EMs; both timed legs below
start at the same phase and run the same K steps.  With --gpus N each rank
analyses its own chip-sized ZMW range (weak scaling, no data exchange).

  value : ZMW-frames/s with the chunks already in HBM
  e2e   : the same K steps through hw_chunk_fused with every step's chunk
          copied from pinned host memory and its results copied back inside
          the timed region: every ZMW's pulse and overflow counts, the valid
          pulse records (packed by hw_pulses_compact; --e2e-download slots
          copies every slot instead) and the HF metrics blocks; copies on
          their own streams, pipelined over pool groups whose engines run on
          two streams (the first upload and the last download overlap nothing)

--impl reference times the oracle (the CPU restatement of the reference's
Host* path) on the host cores over a lane sample of the same workload, with
traces from the oracle's host copy of the generator: nothing of the CUDA
library is loaded on that arm.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hw|reference]
       python bench.py --next-rows    (the stages after and before the chain:
           HF metrics, ingest repacking, BAZ encoding, preliminary HQ -- each
           timed on the GPU and its CPU restatement on a bounded sample)
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FRAMES = 512
LANES_PER_POOL = 4096
POOLS = 4
WORKLOAD = ("chip: 1,048,576 ZMWs (16,384 lanes, 4 pools) x 512-frame int16 chunks, trace generator "
            "workload 1, reference default parameters, dynamic DME")
KERNELS_PER_STAGE = {"baseline": 1, "aggregate": 1, "histogram": 1, "model_init": 1, "dme": 1,
                     "hist_reset": 2, "labeler": 2, "pulses": 1, "metrics": 1}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["hw", "reference"], default="hw")
    ap.add_argument("--lanes-per-pool", type=int, default=LANES_PER_POOL)
    ap.add_argument("--pools", type=int, default=POOLS)
    ap.add_argument("--cpu-lanes", type=int, default=512, help="lanes in the CPU-baseline sample")
    ap.add_argument("--cpu-steps", type=int, default=8)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--next-rows", action="store_true",
                    help="time the HF metrics, repacking, BAZ and preliminary HQ stages, GPU and CPU")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--overlap", type=int, default=1, choices=[0, 1, 2],
                    help="fused engine's use of its second stream (hw_fused_set_overlap)")
    ap.add_argument("--e2e-buffers", type=int, default=3,
                    help="device input/output buffers per group in the end-to-end leg")
    ap.add_argument("--groups", type=int, default=4,
                    help="fused engines the pools are split over (pool groups; both legs, and the end-to-end "
                         "leg pipelines its copies over them)")
    ap.add_argument("--split", type=int, default=1,
                    help="engines each pool's lanes are split over (same pool id, so the same schedule)")
    ap.add_argument("--streams", type=int, default=4,
                    help="streams the group engines run on (group u on stream u mod n)")
    ap.add_argument("--e2e-download", choices=["packed", "slots"], default="packed",
                    help="end-to-end leg's pulse download: the valid records packed by hw_pulses_compact, "
                         "or every pulse slot")
    ap.add_argument("--no-learned-init", action="store_true",
                    help="skip the learned DME initializer measurement (config 3)")
    ap.add_argument("--no-other-configs", action="store_true",
                    help="skip the uneven-pool (config 2) and streaming (config 4) measurements")
    ap.add_argument("--engine", choices=["fused", "analyzers"], default="fused",
                    help="fused: all pools through hw_chunk_fused; analyzers: one hw_analyzer per pool")
    return ap.parse_args()


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def startup_chunks(cfg, pools):
    from hw_b200.workloads import startup_chunks as sc
    return sc(cfg, pools, FRAMES)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5], f[6], f[7], f[8]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return None
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "samples": len(rows), "reasons": sorted(reasons)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return None


def labeler_dram_profile():
    """DRAM bytes per ZMW-frame of the labeler kernel from the committed ncu summary."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "labeler_dram.json")))
        return d
    except Exception:
        return None


def labeler_alg_bytes_per_zmw(F):
    # trace read 2F, labels written 2F, latent traces r+w 2x48, previous model
    # r+w 2x32, boundary label/ROI/latent frame r+w 2x6, new model read 32,
    # LatentTrace output 48, viterbi score 4.
    return 4 * F + 96 + 64 + 12 + 32 + 48 + 4


def cpu_baseline(cfg, lanes, steps, warmup, threads, pools=1, lanes_per_pool=0):
    """The oracle (CPU restatement of the reference Host* path) on a sample of
    lanes of the chip workload, traces from the oracle's host generator (the
    CUDA library is not loaded).  The sample's lanes are split over `pools`
    pools with the GPU run's pool ids, each the first lanes of that pool's
    ZMW range (`lanes_per_pool` lanes a pool on the GPU), and it times the
    same chunks: every step then carries the same share of DME estimates as
    the GPU's, whatever the step count.  Returns (ZMW-frames/s, seconds timed)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hw_b200 import workloads
    oracle.set_threads(threads)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from harness import OracleBackend, Pipeline
    pools = max(1, min(pools, lanes))
    split = [lanes // pools + (1 if p < lanes % pools else 0) for p in range(pools)]
    stage_s = {}
    timing = [False]

    class Timed:
        """The oracle backend with each stage call timed (wall clock)."""
        STAGE = {"baseline": "baseline", "agg_add": "aggregate", "agg_get": "aggregate", "agg_reset": "aggregate",
                 "hist_reset": "hist_reset", "hist_add": "histogram", "hist_get": "histogram",
                 "init_models": "model_init", "estimate": "dme", "label": "labeler", "pulses": "pulses"}

        def __init__(self, b):
            self._b = b
            self.lanes, self.F = b.lanes, b.F

        def startup_latency(self):
            return self._b.startup_latency()

        def __getattr__(self, name):
            fn = getattr(self._b, name)
            stage = Timed.STAGE.get(name)
            if stage is None:
                return fn

            def call(*a):
                t0 = time.perf_counter()
                r = fn(*a)
                if timing[0]:
                    stage_s[stage] = stage_s.get(stage, 0.0) + time.perf_counter() - t0
                return r
            return call

    units = []
    for p, lp in enumerate(split):
        backend = Timed(OracleBackend(cfg, lp, FRAMES, p))
        gen = oracle.TraceGenerator(lp, workload=1, zmw_offset=p * lanes_per_pool * 64)
        units.append((Pipeline(backend, cfg, p), gen))
    n0 = workloads.startup_chunks(cfg, pools, FRAMES, latency=units[0][0].bl_latency) + warmup
    total = n0 + steps
    t_timed = 0.0
    for c in range(total):
        chunks = [gen.next(c * FRAMES, FRAMES) for _, gen in units]
        timing[0] = c >= n0
        t0 = time.perf_counter()
        for (pipe, _), chunk in zip(units, chunks):
            pipe.process(chunk, c * FRAMES)
        dt = time.perf_counter() - t0
        if c >= n0:
            t_timed += dt
    zf = lanes * 64 * FRAMES * steps
    stages = {k: {"ms_per_step": v * 1e3 / steps, "zmw_frames_per_s": zf / v if v > 0 else None}
              for k, v in stage_s.items()}
    return zf / t_timed, t_timed, stages


def next_rows(threads):
    """The four stages beside the chain, each on the GPU (CUDA events, chip
    sizes) and as the CPU restatement (the oracle, one host thread: these
    restatements are sequential, on a bounded sample of the same inputs).
    One JSON line."""
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    from hw_b200 import abi, filters as Fl, workloads
    from hw_b200 import baz as bazm, prehq as prehqm, repack as repackm
    oracle.set_threads(threads)
    out = {"metric": "next rows: GPU and CPU rates", "cpu_cores": 1}
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    # HF metrics on the chain's own chunk outputs (a 4096-lane pool, small configuration)
    lanes, F = 4096, FRAMES
    cfg = workloads.small_config()
    an = Fl.BatchAnalyzer(cfg, 0, lanes, F)
    gen = Fl.TraceGenerator(lanes, workload=1)
    cart = dict(np.load(os.path.join(ROOT, "hw_b200", "data", "trained_cart.npz")))
    inputs = []
    for c in range(16):
        pulses, lens, ovf, em, est = an(gen.next(c * F, F), c * F)
        if em:
            bs, vit, pd = an.chunk_metrics()
            models, _ = an.models()
            inputs.append((pulses.clone(), lens.clone(), bs.clone(), models.clone(), vit.clone(), pd.clone(),
                           c * F - abi.LATENT_FRAMES))
    cap = cfg.max_calls_per_zmw
    hf = Fl.HfMetrics(lanes, 4096, cfg.frame_rate, True, cart=cart)
    for x in inputs[:2]:
        hf.process(x[0], x[1], cap, *x[2:6], x[6], F)
    torch.cuda.synchronize()
    ev0.record()
    for x in inputs[2:]:
        hf.process(x[0], x[1], cap, *x[2:6], x[6], F)
    ev1.record()
    ev1.synchronize()
    n = len(inputs) - 2
    gpu_rate = lanes * 64 * F * n / (ev0.elapsed_time(ev1) / 1e3)
    sl = lanes   # CPU sample: the whole pool
    ref = oracle.HfMetrics(sl, 4096, cfg.frame_rate, True)
    ref.set_cart(cart)
    host = [(Fl.struct_to_numpy(x[0], abi.PULSE_DT).reshape(lanes, 64, cap)[:sl].copy(),
             x[1].cpu().numpy().astype(np.uint32).reshape(lanes, 64)[:sl].copy(),
             Fl.struct_to_numpy(x[2], abi.BLSTATS_DT)[:sl].copy(), Fl.struct_to_numpy(x[3], abi.LANE_MODEL_DT)[:sl].copy(),
             x[4].cpu().numpy().reshape(lanes, 64)[:sl].copy(), Fl.struct_to_numpy(x[5], abi.STAT_ACCUM_DT)[:sl].copy(),
             x[6]) for x in inputs]
    t0 = time.perf_counter()
    for h in host:
        ref.process(*h[:6], h[6], F)
    cpu_s = time.perf_counter() - t0
    out["hf_metrics"] = {"unit": "ZMW-frames/s", "gpu": gpu_rate,
                         "cpu": sl * 64 * F * len(host) / cpu_s,
                         "gpu_workload": f"{lanes} lanes, {n} chunks of {F} frames of the chain's outputs",
                         "cpu_sample": f"{sl} lanes, {len(host)} chunks ({cpu_s:.2f} s)"}
    del an, inputs, host

    # ingest repacking: the chip chunk on the GPU; 16,384 ZMWs of it on the CPU
    r = repackm.run(steps=10)
    nz_s = 131072
    table, nbytes = repackm.chip_packets(nz_s, F)
    data = np.random.default_rng(1).integers(0, 255, nbytes, dtype=np.uint8)
    chunks = [np.zeros((nz_s // 64, F, 64), np.int16)]
    t0 = time.perf_counter()
    for _ in range(10):
        oracle.repack(nz_s, nz_s // 64, F, 0, table, data, 0, chunks)
    cpu_s = (time.perf_counter() - t0) / 10
    out["repack"] = {"unit": "ZMW-frames/s", "gpu": r["zmw_frames_per_s"], "cpu": nz_s * F / cpu_s,
                     "gpu_workload": r["workload"], "cpu_sample": f"{nz_s} ZMWs x {F} frames ({cpu_s:.3f} s a chunk)"}

    # BAZ encoding: consecutive chip chunks on the GPU; 32,768 ZMWs of them on the CPU
    b = bazm.run(steps=5, warmup=3)
    pool_chunks, cap = bazm.chain_pulses(3)
    nz_s = 262144
    fields, skip = Fl.baz_preset(abi.BAZ_PRODUCTION)
    enc = oracle.BazEncoder(fields, skip, nz_s)
    host = [(Fl.struct_to_numpy(p, abi.PULSE_DT).reshape(-1, cap)[:nz_s].copy(),
             l.cpu().numpy().astype(np.uint32).reshape(-1)[:nz_s].copy()) for p, l in pool_chunks]
    t0 = time.perf_counter()
    npul = 0
    for p, l in host:
        enc(p, l, cap)
        npul += int(l.sum())
    cpu_s = time.perf_counter() - t0
    nz_s = 32768
    host = [(p[:nz_s].copy(), l[:nz_s].copy()) for p, l in host]
    out["baz_encoding"] = {"unit": "pulses/s", "gpu": b["pulses_per_s"], "cpu": npul / cpu_s,
                           "gpu_workload": b["workload"], "cpu_sample": f"262144 ZMWs x {len(host)} chunks, "
                                                                        f"{npul} pulses ({cpu_s:.2f} s)"}

    # preliminary HQ: the chip stage on the GPU; 32,768 ZMWs through encoding + stage on the CPU
    q = prehqm.run(blocks=2, warmup_blocks=11)
    st = oracle.PrelimHq(nz_s, 10, True, 0.10)
    enc = oracle.BazEncoder(fields, skip, nz_s)
    t0 = time.perf_counter()
    nchunks = 0
    for blk in range(13):
        for c in range(8):
            p, l = host[(blk * 8 + c) % len(host)]
            d, off = enc(p, l, cap)
            kept = (np.minimum(l, cap)[:, None] > np.arange(cap)[None, :]) & (p["is_reject"] == 0)
            st.add(d, off, kept.sum(axis=1).astype(np.uint32))
            nchunks += 1
        st.end_block()
    cpu_s = time.perf_counter() - t0
    out["prelim_hq"] = {"unit": "ZMW-frames/s", "gpu": q["zmw_frames_per_s"], "cpu": nz_s * F * nchunks / cpu_s,
                        "gpu_workload": q["workload"],
                        "cpu_sample": f"{nz_s} ZMWs x {nchunks} chunks, encoding included ({cpu_s:.2f} s)"}
    print(json.dumps(out))


def main():
    args = parse()
    world, rank, local = dist_setup()
    from hw_b200 import workloads
    cfg = workloads.chip_config()
    total_lanes = args.lanes_per_pool * args.pools
    zmws = total_lanes * 64
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        # The reference path on the host cores: rank 0 alone, no CUDA and no
        # collective (the other ranks exit at once).
        if rank == 0:
            rate, secs, stages = cpu_baseline(cfg, args.cpu_lanes, max(args.steps, 1), args.warmup, threads,
                                              args.pools, args.lanes_per_pool)
            sample = (f"{args.cpu_lanes} lanes ({args.cpu_lanes * 64} ZMWs) of the workload, spread over its "
                      f"{args.pools} pools, x {args.steps} steady-state 512-frame chunks after start-up "
                      f"(the GPU run's chunks), {secs:.1f} s of CPU time")
            zf_step = args.cpu_lanes * 64 * FRAMES
            out = {"metric": "ZMW-frames/s", "value": rate, "unit": "ZMW-frames/s", "impl": "reference",
                   "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                   "ms_per_step": zf_step / rate * 1e3, "higher_is_better": True, "scaling": "weak",
                   "vs_baseline": None, "dtype": "int16+f32", "data": "synthetic",
                   "config": {"workload": WORKLOAD, "zmws_per_gpu": zmws, "frames_per_chunk": FRAMES,
                              "pools": args.pools, "cpu_sample_lanes": args.cpu_lanes},
                   "cpu_baseline": {"value": rate, "unit": "ZMW-frames/s", "cores": threads, "kind": "port",
                                    "sample": sample, "stages": stages},
                   "e2e": {"value": rate, "unit": "ZMW-frames/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}}
            print(json.dumps(out), flush=True)
        return

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from hw_b200 import filters as Fl
    if args.next_rows:
        if rank == 0:
            next_rows(os.cpu_count() or 1)
        return

    from hw_b200.shard import zmw_offset
    gen = Fl.TraceGenerator(total_lanes, workload=1, zmw_offset=zmw_offset(rank, zmws))
    lpp = args.lanes_per_pool
    stream = torch.cuda.current_stream()
    serial = [False]
    if args.engine == "fused":
        # The pools in G groups, one engine each (a group keeps its pools' ids
        # and so their estimation stagger): each stage is one launch over the
        # lanes of a group's pools, HF metrics included (4096-frame blocks,
        # the reference's trained activity classifier).  The engines run on
        # NS streams, so one group's DME (a latency-bound launch) shares the
        # GPU with other groups' stages.
        # With --split S each pool's lanes form S sub-pools of lpp / S lanes
        # that keep the pool's id (lanes are independent, and the schedule
        # depends on the id only); below, "pools" of an engine are sub-pools.
        SP = max(1, args.split) if lpp % max(1, args.split) == 0 else 1
        ul = lpp // SP
        nsub = args.pools * SP
        G = max(1, min(args.groups * SP, nsub))
        if nsub % G:
            G = 1
        ppg = nsub // G
        NS = max(1, min(args.streams, G))
        cart = dict(np.load(os.path.join(ROOT, "hw_b200", "data", "trained_cart.npz")))
        engines = []
        for g in range(G):
            ids = list(range(g * ppg, (g + 1) * ppg))
            eg = Fl.FusedEngine(cfg, [ul] * ppg, [FRAMES] * ppg, pool_ids=[i // SP for i in ids])
            eg.set_overlap(args.overlap)
            eg.enable_hf_metrics(4096, cfg.frame_rate, True, cart)
            engines.append((eg, ids))
        s_comp = [stream] + [torch.cuda.Stream() for _ in range(NS - 1)]
        profiled = [eg for eg, _ in engines]
        outputs = [engines[p // ppg][0].outputs(p % ppg) for p in range(nsub)]
        pool_metrics = [eg.metrics[i] for eg, ids in engines for i in range(len(ids))]

        def run_units(chunk, outs=None):
            for u, (eg, ids) in enumerate(engines):
                with torch.cuda.stream(stream if serial[0] else s_comp[u % NS]):
                    eg.process([chunk[p * ul:(p + 1) * ul] for p in ids], outs[u] if outs else None)
    else:
        G, NS, s_comp, ul, SP = args.pools, 1, [stream], lpp, 1
        analyzers = [Fl.BatchAnalyzer(cfg, p, lpp, FRAMES) for p in range(args.pools)]
        profiled = analyzers
        outputs = [(a.pulses, a.lens, a.ovf) for a in analyzers]

        def run_units(chunk, c, outs=None):
            for p, a in enumerate(analyzers):
                o = outs[p] if outs is not None else (None, None, None)
                a(chunk[p * lpp:(p + 1) * lpp], c * FRAMES, *o)

    def fork():
        for s_ in s_comp[1:]:
            s_.wait_stream(stream)

    def join():
        for s_ in s_comp[1:]:
            stream.wait_stream(s_)

    def run_chunk(chunk, c, sync=True):
        # sync: the chunk buffer is reused by the caller's next step
        if sync:
            fork()
        if args.engine == "fused":
            run_units(chunk)
        else:
            run_units(chunk, c)
        if sync:
            join()

    # Start-up and warm-up (untimed).
    n_start = startup_chunks(cfg, args.pools)
    buf = torch.empty((total_lanes, FRAMES, 64), dtype=torch.int16, device="cuda")
    c = 0
    for _ in range(n_start + args.warmup):
        gen.next(c * FRAMES, FRAMES, out=buf)
        run_chunk(buf, c)
        c += 1
    torch.cuda.synchronize()

    # Device-resident timed region.
    K = args.steps
    c_dev0 = c
    dev_chunks = []
    for k in range(K):
        t = torch.empty((total_lanes, FRAMES, 64), dtype=torch.int16, device="cuda")
        gen.next((c + k) * FRAMES, FRAMES, out=t)
        dev_chunks.append(t)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    from hw_b200.shard import max_over_ranks

    clocks = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    fork()
    for k in range(K):
        run_chunk(dev_chunks[k], c + k, sync=False)
    join()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    c += K
    # Stage times from a second pass over the same chunks (the next K frames:
    # again one full estimation cycle) with the stage timers on; untimed, so
    # the timers' events do not weigh on the rate above.
    for a in profiled:
        a.profile(True)
        a.stage_times()
    serial[0] = True        # one stream: the stage timers time the stream they run on
    for k in range(K):
        run_chunk(dev_chunks[k], c + k)
    torch.cuda.synchronize()
    serial[0] = False
    c += K
    del dev_chunks
    stage = {}
    for a in profiled:
        for kname, (t_ms, n) in a.stage_times().items():
            s = stage.setdefault(kname, [0.0, 0])
            s[0] += t_ms
            s[1] += n
        a.profile(False)
    launches = sum(n * KERNELS_PER_STAGE[k] for k, (_, n) in stage.items())
    if args.engine == "fused":
        launches += 2 * K * G      # per step and engine: the step-table upload and the failure-word kernels

    zf_step = zmws * FRAMES
    value = zf_step * K * world / (ms / 1e3)

    # End-to-end through the C ABI: every step copies its chunk from pinned
    # host memory to the device, analyses it and copies its results back to
    # pinned host memory.  Copies run on their own streams, buffered against
    # the analysis: step k's upload and step k-1's download overlap step k's
    # kernels.
    e2e = None
    if not args.no_e2e:
        # The same K steps from the same phase of the estimation cycle as
        # the device-resident leg (so both run the same number of EMs): the
        # engine first streams untimed chunks up to that phase.  Up to 16
        # distinct pinned chunks are uploaded in turn (every step still moves
        # its 1 GiB).
        cycle = (max(int(cfg.min_frames_for_estimate), 1) + FRAMES - 1) // FRAMES
        while (c - c_dev0) % cycle:
            gen.next(c * FRAMES, FRAMES, out=buf)
            run_chunk(buf, c)
            c += 1
        torch.cuda.synchronize()
        KE = K
        # Copy/compute pipelining over the pool groups: each group's chunk
        # slice is uploaded, analysed by its engine and downloaded on its
        # own, so a step's first upload and last download cover one group,
        # not the whole chip.
        if args.engine == "fused":
            units = engines
        else:
            units = [(analyzers[p], [p]) for p in range(args.pools)]
        ppg = len(units[0][1])

        def run_unit(u, chunk_slice, outs):
            eg, ids = units[u]
            if args.engine == "fused":
                eg.process([chunk_slice[i * ul:(i + 1) * ul] for i in range(len(ids))], outs)
            else:
                eg(chunk_slice, (c + k) * FRAMES, *outs[0])

        host_chunks = []
        tmp = torch.empty((total_lanes, FRAMES, 64), dtype=torch.int16, device="cuda")
        for k in range(min(KE, 16)):
            gen.next((c + k) * FRAMES, FRAMES, out=tmp)
            h = torch.empty((total_lanes, FRAMES, 64), dtype=torch.int16, pin_memory=True)
            h.copy_(tmp)
            host_chunks.append(h)
        del tmp
        U = len(units)
        NB = max(2, args.e2e_buffers)    # input and output buffers per group: copies may run NB - 1 steps ahead
        rows = [(units[u][1][0] * ul, (units[u][1][-1] + 1) * ul) for u in range(U)]
        in_dev = [[torch.empty((r1 - r0, FRAMES, 64), dtype=torch.int16, device="cuda") for r0, r1 in rows]
                  for _ in range(NB)]
        out_dev = [[[(torch.empty_like(outputs[p][0]), torch.empty_like(outputs[p][1]),
                      torch.empty_like(outputs[p][2])) for p in units[u][1]] for u in range(U)] for _ in range(NB)]
        host_out = [(torch.empty(dp.numel(), dtype=torch.uint8, pin_memory=True),
                     torch.empty(dl.shape, dtype=torch.int32, pin_memory=True),
                     torch.empty(do.shape, dtype=torch.int32, pin_memory=True)) for dp, dl, do in outputs]
        hf_host = ([torch.empty(m.numel(), dtype=torch.uint8, pin_memory=True) for m in pool_metrics]
                   if args.engine == "fused" else [])
        metrics_bytes = 0
        # Packed download: hw_pulses_compact packs each pool's valid records
        # after the analysis, and the host copies exactly that many bytes.
        # The count is read from the compactor's mapped slot once the group's
        # analysis has passed, a few groups after it was queued (the host
        # stays that far ahead of the device), so the copy of those records
        # is queued then.
        packed = args.e2e_download == "packed"
        max_calls = int(cfg.max_calls_per_zmw)
        rec_bytes = outputs[0][0].numel() // (outputs[0][1].numel() * max_calls)
        if packed:
            compactors = [Fl.PulseCompactor(dl.numel()) for _, dl, _ in outputs]
            packed_dev = [[[(torch.empty_like(outputs[p][0]),
                             torch.empty(outputs[p][1].numel() + 1, dtype=torch.int64, device="cuda"))
                            for p in units[u][1]] for u in range(U)] for _ in range(NB)]
        pending = []
        # a compactor's two count slots alternate per call, so a group's
        # count is read before that engine's call two steps later is queued
        DEFER = max(1, 2 * U - 1)
        record_bytes = 0

        def download_records(b_, u_, slots_):
            # on a stream of their own: queued behind the next groups'
            # count copies, which wait for those groups' analysis, they
            # would pile up to the end of the run
            ev_comp[b_][u_].synchronize()
            n_bytes = 0
            with torch.cuda.stream(s_rec):
                s_rec.wait_event(ev_small[b_][u_])
                for p, (co, _), sl in zip(units[u_][1], packed_dev[b_][u_], slots_):
                    nb_ = compactors[p].total(sl) * rec_bytes
                    if nb_:
                        host_out[p][0][:nb_].copy_(co.view(-1)[:nb_], non_blocking=True)
                    n_bytes += nb_
                ev_d2h[b_][u_].record(s_rec)
            return n_bytes
        s_h2d, s_d2h = torch.cuda.Stream(), torch.cuda.Stream()
        s_mark = torch.cuda.Stream()
        s_rec = torch.cuda.Stream()         # the packed records' copies, queued late
        ev_small = [[torch.cuda.Event() for _ in range(U)] for _ in range(NB)]
        ev_h2d = [[torch.cuda.Event() for _ in range(U)] for _ in range(NB)]
        ev_comp = [[torch.cuda.Event() for _ in range(U)] for _ in range(NB)]
        ev_d2h = [[torch.cuda.Event() for _ in range(U)] for _ in range(NB)]
        ev_step = [torch.cuda.Event(enable_timing=True) for _ in range(KE)]
        if packed:
            # load the compaction kernels before the timed region
            for u in range(U):
                for p, (dp, dl, _), (co, off) in zip(units[u][1], out_dev[0][u], packed_dev[0][u]):
                    compactors[p].total(compactors[p](dp, dl, max_calls, co, off))
        torch.cuda.synchronize()
        barrier()
        e0.record(stream)
        for s_ in [s_h2d, s_d2h, s_mark, s_rec] + s_comp[1:]:
            s_.wait_stream(stream)
        for k in range(KE):
            b = k % NB
            src = host_chunks[k % len(host_chunks)]
            for u in range(U):
                r0, r1 = rows[u]
                su = s_comp[u % NS]
                with torch.cuda.stream(s_h2d):
                    if k >= NB:
                        s_h2d.wait_event(ev_comp[b][u])     # step k-NB has read in_dev[b][u]
                    in_dev[b][u].copy_(src[r0:r1], non_blocking=True)
                    ev_h2d[b][u].record(s_h2d)
                su.wait_event(ev_h2d[b][u])
                if k >= NB:
                    su.wait_event(ev_d2h[b][u])             # step k-NB's outputs are on the host
                with torch.cuda.stream(su):
                    run_unit(u, in_dev[b][u], out_dev[b][u])
                    slots = ([compactors[p](dp, dl, max_calls, co, off)
                              for p, (dp, dl, _), (co, off) in zip(units[u][1], out_dev[b][u], packed_dev[b][u])]
                             if packed else None)
                ev_comp[b][u].record(su)
                s_mark.wait_event(ev_comp[b][u])
                with torch.cuda.stream(s_d2h):
                    s_d2h.wait_event(ev_comp[b][u])
                    for p, (dp, dl, do) in zip(units[u][1], out_dev[b][u]):
                        hp, hl, ho = host_out[p]
                        hl.copy_(dl, non_blocking=True)
                        ho.copy_(do, non_blocking=True)
                        if not packed:
                            hp.copy_(dp, non_blocking=True)
                            record_bytes += dp.numel()
                    if args.engine == "fused":
                        # HF metrics records of the pools that completed a block
                        eg = units[u][0]
                        for i, em in enumerate(eg.metrics_emitted()):
                            if em:
                                p = units[u][1][i]
                                hf_host[p].copy_(eg.metrics[i], non_blocking=True)
                                metrics_bytes += eg.metrics[i].numel()
                    if packed:
                        ev_small[b][u].record(s_d2h)
                    else:
                        ev_d2h[b][u].record(s_d2h)
                if packed:
                    pending.append((b, u, slots))
                    while len(pending) > DEFER:
                        record_bytes += download_records(*pending.pop(0))
            ev_step[k].record(s_mark)                       # every group of step k analysed
        while pending:
            record_bytes += download_records(*pending.pop(0))
        for s_ in [s_d2h, s_mark, s_rec] + s_comp[1:]:
            stream.wait_stream(s_)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1))
        # where the time went: the analysis of step k ends at ev_step[k]
        marks = [e0.elapsed_time(ev) for ev in ev_step]
        timeline = {"first_step_done_ms": marks[0],
                    "step_ms_after_first": [b_ - a_ for a_, b_ in zip(marks, marks[1:])],
                    "last_download_ms": ms_e2e - marks[-1]}
        # untimed check: the host holds the last step's results (counts, and
        # the packed records or every slot) as they are on the device
        bl = (KE - 1) % NB
        verified = True
        for u in range(U):
            for j, p in enumerate(units[u][1]):
                dp, dl, do = out_dev[bl][u][j]
                hp, hl, ho = host_out[p]
                verified &= torch.equal(hl, dl.cpu()) and torch.equal(ho, do.cpu())
                if packed:
                    co, off = packed_dev[bl][u][j]
                    nb_ = int(off[-1].item()) * rec_bytes
                    verified &= torch.equal(hp[:nb_], co.view(-1)[:nb_].cpu())
                else:
                    verified &= torch.equal(hp, dp.cpu())
        c += KE
        h2d = total_lanes * FRAMES * 64 * 2
        d2h = (record_bytes + metrics_bytes) // KE + sum(dl.numel() * 4 + do.numel() * 4 for _, dl, do in outputs)
        e2e = {"value": zf_step * KE * world / (ms_e2e / 1e3), "unit": "ZMW-frames/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": ms_e2e / KE, "steps": KE,
               "phase": "same K steps of the estimation cycle as value", "timeline": timeline,
               "verified": bool(verified),
               "overlap": f"copies on their own streams, {NB} buffers deep against the analysis, pipelined over "
                          f"{U} pool group(s) of {ppg * ul} lanes (one engine each, on {NS} stream(s)); a step's "
                          f"first upload and last download cover one group",
               "download": ("the valid pulse records, packed by hw_pulses_compact, with every ZMW's pulse and "
                            "overflow counts and the HF metrics blocks" if packed else
                            "every pulse slot, with every ZMW's pulse and overflow counts and the HF metrics blocks")}
        if packed:
            for cp in compactors:
                cp.close()
            del packed_dev
        del host_chunks, in_dev, out_dev

    # Roofline of the dominant kernel (the frame labeler) from the live stage timers.
    peaks = measured_peaks()
    lab_ms, lab_n = stage.get("labeler", (0.0, 0))
    roof = None
    if lab_n:
        # the stage pass labels every ZMW once a step, in launches of
        # different sizes (a step with an estimate labels the estimating
        # pools in a launch of their own): bytes and time are totals over
        # the pass, per launch their averages
        zmw_labeled = zmws * K
        lab_bytes_launch = labeler_alg_bytes_per_zmw(FRAMES) * zmw_labeled / lab_n
        achieved = labeler_alg_bytes_per_zmw(FRAMES) * zmw_labeled / (lab_ms / 1e3) / 1e9
        peak = peaks["hbm_gbs"] if peaks else 6650.0
        prof = labeler_dram_profile()
        traffic = None
        if prof:
            traffic = prof["dram_bytes_per_zmw_frame"] * zmw_labeled * FRAMES / lab_n
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic,
                "kernel": "LabelerKernel", "launch_ms": lab_ms / lab_n,
                "alg_bytes_per_launch": lab_bytes_launch,
                "peak_source": "measured" if peaks else "fallback"}
        if prof and "issue_frac" in prof:
            roof["issue_roofline"] = {"frac": prof["issue_frac"],
                                      "source": "ncu smsp__issue_active of the labeler, small case"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, secs, stages = cpu_baseline(cfg, args.cpu_lanes, args.cpu_steps, args.warmup, threads,
                                          args.pools, args.lanes_per_pool)
        cpu = {"value": rate, "unit": "ZMW-frames/s", "cores": threads, "kind": "port", "stages": stages,
               "sample": f"{args.cpu_lanes} lanes ({args.cpu_lanes * 64} ZMWs) spread over the {args.pools} "
                         f"pools x {args.cpu_steps} steady-state 512-frame chunks after start-up ({secs:.1f} s)"}

    if args.engine == "fused":
        for eg, _ in engines:
            eg.finish()
    for a in profiled:
        a.close()
    learned = None
    net = None
    if rank == 0 and world == 1 and not args.no_learned_init:
        # BASELINE metric part 2: EM iterations from the learned start vs the
        # plain start (2.1M training ZMWs of the uneven-pool generator,
        # 262K held-out ZMWs), measured after the timed regions.
        from hw_b200 import learned_init
        t0 = time.time()
        net, learned = learned_init.run()
        learned["seconds"] = time.time() - t0
        ph = learned.get("dme_phases", {})
        if ph:
            learned["dme_stage_ms_4096_lanes"] = {
                "plain_start": ph["plain"]["estimate_ms"],
                "learned_start": ph["learned"]["network_ms"] + ph["learned"]["estimate_ms"]}

    other = None
    if rank == 0 and world == 1 and not args.no_other_configs:
        # the other single-GPU configurations, after the timed regions: uneven
        # pools through the tuned fused engine, and the streaming run with
        # the reference start and (when trained above) the learned start
        from hw_b200 import streaming, uneven, workloads
        other = {}
        t0 = time.time()
        u = uneven.run(variants=("fused_tuned",))
        other["uneven_pools"] = {k: u[k] for k in ("pools", "zmws", "lanes_min", "lanes_max", "chunk_lengths",
                                                   "timed_steps", "warmup_steps", "fused_tuned_ms_per_step",
                                                   "fused_tuned_zmw_frames_per_s", "fused_tuned_launches_per_step")}
        other["uneven_pools"]["workload"] = ("500 pools, lanes log-uniform in [1, 2048], chunks of 128/256/512 "
                                             "frames, uneven-pool generator, dynamic DME")
        other["uneven_pools"]["seconds"] = time.time() - t0
        t0 = time.time()
        scfg = workloads.chip_config()
        st = {"workload": "streaming: 2,097,152 ZMWs (8 pools of 4096 lanes) x 128 chunks of 512 frames, "
                          "generated on the GPU (decay 20%, +15 DN step in 1% of ZMWs), dynamic DME; one "
                          "one-pool fused engine per pool, on four streams (stage times from the same run on "
                          "one stream)",
              "plain_em": streaming.run_chain(scfg, 8, 4096, 128, streams=4, engine="fused"),
              "one_stream": {"plain_em": streaming.run_chain(scfg, 8, 4096, 128, engine="fused")}}
        if net is not None:
            st["learned_init"] = streaming.run_chain(scfg, 8, 4096, 128, net, streams=4, engine="fused")
            st["one_stream"]["learned_init"] = streaming.run_chain(scfg, 8, 4096, 128, net, engine="fused")
        st["seconds"] = time.time() - t0
        other["streaming"] = st
    if net is not None:
        net.close()

    if rank == 0:
        out = {
            "metric": "ZMW-frames/s", "value": value, "unit": "ZMW-frames/s", "n_gpus": world,
            "steps": K, "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16+f32", "data": "synthetic",
            "config": {"workload": WORKLOAD,
                       "zmws_per_gpu": zmws, "frames_per_chunk": FRAMES, "pools": args.pools,
                       "startup_chunks": n_start, "inputs": "1 GiB chunk per step, larger than L2",
                       "engine": (f"hw_chunk_fused: {G} engine(s) of {ppg} pool(s) of {ul} lanes (one launch per "
                                  f"stage over an engine's pools{'; each pool split over %d engines' % SP if SP > 1 else ''}) "
                                  f"on {NS} stream(s)" if args.engine == "fused"
                                  else "one hw_analyzer per pool")},
            "e2e": e2e, "gpu_launches": launches, "roofline": roof, "cpu_baseline": cpu,
            "clocks": clk,
            "stage_ms": {k: v[0] / K for k, v in stage.items()},
            "learned_init": learned,
            "other_configs": other,
        }
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
