"""hw_b200: B200-native smrt-basecaller trace-analysis chain.

Baseline filter -> trace histogram -> detection-model EM -> frame labeling ->
pulse accumulation, as sm_100a CUDA kernels behind a C ABI
(include/hw_b200.h, libhw_b200.so), with host mirrors of the reference's
per-pool filter interfaces.
"""
from . import abi  # noqa: F401

__all__ = ["abi"]
