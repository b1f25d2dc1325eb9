"""yaoray_b200 — B200-native (sm_100a) wavefront path-tracing backend for YaoRay.

The compute path is libyrcuda (hand-written CUDA kernels behind the C ABI in
include/yrcuda.h); this package is the Python host mirror of the reference's
accel / backend interfaces used by the tests and the benchmark.
"""
from ._lib import YrcError, lib  # noqa: F401

__version__ = "0.1.0"
