"""scycle_b200: SCycle's per-time-step quasi-dynamic path on NVIDIA B200 (sm_100a).

The compute path is libscycle_b200.so (hand-written CUDA behind a C ABI,
include/scycle_b200.h).  This package holds the build step, the ctypes
binding and thin Python mirrors of the reference classes used by tests and
the benchmark.
"""
__all__ = ["build", "configs"]
