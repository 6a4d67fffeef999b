"""The whole path (hw_b200.pipeline: repacking -> fused engine with HF
metrics -> BAZ encoding + preliminary HQ) against the same path composed
stage by stage: per-pool analyzers on the traces, then the oracle's BAZ
encoder and preliminary HQ stage.  Every checkpoint equal byte for byte."""
import numpy as np
import pytest

from hw_b200 import abi


@pytest.mark.gpu
@pytest.mark.parametrize("streams", [1, 2])
def test_pipeline_checkpoints_equal_stage_by_stage(streams):
    """streams = 1: one engine over both pools; 2: an engine per pool, each on
    its own stream with its pool's BAZ / preliminary HQ stage."""
    import torch
    import oracle
    from hw_b200 import filters as Fl, pipeline, workloads
    cfg = workloads.small_config()
    pools, lanes, F, n_inputs = 2, 32, pipeline.F, 8
    got = []
    pipeline.run(steps=16, warmup_steps=8, n_inputs=n_inputs, pools=pools, lanes=lanes, cfg=cfg, collect=got,
                 streams=streams)
    assert len(got) >= 2 * pools
    # the same traces: the generator's first n_inputs chunks, used in turn
    gen = Fl.TraceGenerator(pools * lanes, workload=1)
    traces = [gen.next(c * F, F).clone() for c in range(n_inputs)]
    fields, skip = Fl.baz_preset(abi.BAZ_PRODUCTION)
    cap = cfg.max_calls_per_zmw
    nz = lanes * 64
    want = {}
    for p in range(pools):
        an = Fl.BatchAnalyzer(cfg, p, lanes, F)
        enc = oracle.BazEncoder(fields, skip, nz)
        st = oracle.PrelimHq(nz, 10, False)
        added = 0
        for c in range(24):
            chunk = traces[c % n_inputs][p * lanes:(p + 1) * lanes].contiguous()
            pulses, lens, ovf, em, est = an(chunk, c * F)
            if not em:
                continue
            hp = Fl.struct_to_numpy(pulses, abi.PULSE_DT).reshape(nz, cap)
            hl = lens.cpu().numpy().astype(np.uint32).reshape(nz)
            data, off = enc(hp, hl, cap)
            kept = (np.minimum(hl, cap)[:, None] > np.arange(cap)[None, :]) & (hp["is_reject"] == 0)
            st.add(data, off, kept.sum(axis=1).astype(np.uint32))
            added += 1
            if added % 8 == 0:
                want[(c, p)] = st.end_block()
    keys = [(c, p) for c, p, _ in got]
    assert keys == sorted(want, key=lambda k: (k[0], k[1]))
    for c, p, out in got:
        data, off, ev, hq = want[(c, p)]
        assert out["offsets"].cpu().numpy().astype(np.uint64).tolist() == off.tolist(), (c, p)
        assert out["bytes"].cpu().numpy().tobytes() == data.tobytes(), (c, p)
        assert (out["events"].cpu().numpy() == ev).all()
        assert (out["hq"].cpu().numpy() == hq).all()
