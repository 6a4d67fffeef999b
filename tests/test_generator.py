"""The workloads' trace generator: the oracle's host copy (used by the CPU
baseline, so it needs no CUDA library) has the library's workload defaults
and, on the GPU, writes the same bytes as hw_trace_generator for every
workload, over consecutive chunks (pulse state carried across chunks) and
across the streaming workload's amplitude decay and baseline step."""
import ctypes as C

import numpy as np
import pytest

from hw_b200 import abi, native


def _fields(p):
    return [(n, list(getattr(p, n)) if n == "amplitudes" else getattr(p, n)) for n, _ in abi.GenParams._fields_]


@pytest.mark.parametrize("workload", [0, 1, 2, 4])
def test_host_defaults_equal_library_defaults(workload):
    import oracle
    lib = abi.GenParams()
    native.check(native.lib().hw_gen_params_default(workload, C.byref(lib)))
    assert _fields(oracle.gen_params_default(workload)) == _fields(lib)


def test_host_generator_statistics():
    """Chip workload: baseline near 200 DN with sigma 8 plus a random walk,
    pulses on roughly 8 / (8 + 14) of the non-empty ZMWs' frames."""
    import oracle
    g = oracle.TraceGenerator(4, workload=0)
    x = np.concatenate([g.next(c * 512, 512) for c in range(4)], axis=1).astype(np.float64)
    base = x[x < 230]
    assert abs(np.median(base) - 200) < 3 and 6 < base.std() < 12
    assert 0.2 < (x > 215).mean() < 0.45


@pytest.mark.gpu
@pytest.mark.parametrize("workload,first", [(0, 0), (1, 0), (2, 0), (4, 31744)])
def test_host_generator_equals_device(workload, first):
    import torch
    import oracle
    from hw_b200 import filters as Fl
    lanes, F = 3, 512
    dev = Fl.TraceGenerator(lanes, workload=workload, zmw_offset=777)
    host = oracle.TraceGenerator(lanes, workload=workload, zmw_offset=777)
    for c in range(4):
        ff = first + c * F
        a = dev.next(ff, F).cpu().numpy()
        b = host.next(ff, F)
        assert np.array_equal(a, b), (workload, c)
