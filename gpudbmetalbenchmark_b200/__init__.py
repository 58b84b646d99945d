"""gpudbmetalbenchmark_b200 -- B200-native columnar query engine for the hot path of
nd-tung/GPUDBMetalBenchmark: fused filter+aggregate scans, hash-join build/probe with
radix partitioning, bitmap semi-join filters, device top-k and chunked host->HBM
streaming, as sm_100a CUDA kernels behind the C ABI of include/gpudb_capi.h.
"""
from . import capi  # noqa: F401
from .engine import Engine, Table  # noqa: F401

__all__ = ["Engine", "Table", "capi"]
