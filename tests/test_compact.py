"""Pulse compaction (hw_pulses_compact): the valid records of every ZMW,
packed in ZMW order, equal to packing them on the host."""
import numpy as np
import pytest

from hw_b200 import abi


@pytest.mark.gpu
@pytest.mark.parametrize("nz,cap", [(1, 8), (777, 48), (70000, 24)])
def test_gpu_compaction_packs_the_valid_records(nz, cap):
    import torch
    from hw_b200 import filters as Fl
    rng = np.random.default_rng(nz)
    p = np.zeros((nz, cap), abi.PULSE_DT)
    for name in ("start", "width", "mean_signal", "mid_signal", "max_signal", "label", "is_reject"):
        p[name] = rng.integers(0, 200, (nz, cap))
    p["signal_m2"] = rng.random((nz, cap)).astype(np.float32)
    lens = rng.integers(0, cap + 3, nz).astype(np.uint32)     # some counts past the slots
    comp = Fl.PulseCompactor(nz)
    d_p = torch.from_numpy(p.view(np.uint8).reshape(-1).copy()).cuda()
    d_l = torch.from_numpy(lens.view(np.int32)).cuda()
    out = torch.zeros(nz * cap * abi.PULSE_DT.itemsize, dtype=torch.uint8, device="cuda")
    off = torch.zeros(nz + 1, dtype=torch.int64, device="cuda")
    totals = []
    for _ in range(3):   # the slots alternate
        slot = comp(d_p, d_l, cap, out, off)
        torch.cuda.synchronize()
        totals.append(comp.total(slot))
    n = np.minimum(lens, cap)
    want = np.concatenate([p[z, :n[z]] for z in range(nz)]) if n.sum() else np.zeros(0, abi.PULSE_DT)
    assert totals == [int(n.sum())] * 3
    assert off.cpu().numpy().tolist() == np.concatenate([[0], np.cumsum(n)]).tolist()
    got = out.cpu().numpy()[:len(want) * abi.PULSE_DT.itemsize].view(abi.PULSE_DT)
    assert got.tobytes() == want.tobytes()
