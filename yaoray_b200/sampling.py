"""The device's sampling primitives evaluated through the C ABI, for checking
the sample values the path tracer draws against the reference's: the
per-pixel sampler (Sampler, src/sampling/sampler.cpp:122-310), PCG32 (Rng,
include/yaoray/core/rng.hpp:15-48) and SeedForPixelSample
(sampler.cpp:304-310). Each call runs a CUDA kernel on host arrays and
returns host arrays."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib

INDEPENDENT, STRATIFIED, OWEN_SOBOL, Z_SOBOL = 0, 1, 2, 3


def sampler_eval(kind: int, seed: int, spp: int, queries: np.ndarray, two_d: bool) -> np.ndarray:
    """Sample1D (two_d False, shape (n,)) or Sample2D (shape (n, 2)) of the
    sampler `kind` for rows (x, y, sample, bounce, dimension, lane)."""
    q = np.ascontiguousarray(queries, np.int32).reshape(-1, 6)
    out = np.empty(q.shape[0] * (2 if two_d else 1), np.float32)
    _lib.check(_lib.lib().yrc_sampler_eval(int(kind), C.c_uint64(seed), int(spp), _lib.ptr(q), q.shape[0],
                                           int(bool(two_d)), _lib.ptr(out)))
    return out.reshape(-1, 2) if two_d else out


def rng_eval(seeds: np.ndarray, draws: int) -> np.ndarray:
    """`draws` NextFloat values of Rng(seed) for each seed: shape (n, draws)."""
    s = np.ascontiguousarray(seeds, np.uint64).reshape(-1)
    out = np.empty((s.shape[0], int(draws)), np.float32)
    _lib.check(_lib.lib().yrc_rng_eval(_lib.ptr(s), s.shape[0], int(draws), _lib.ptr(out)))
    return out


def pixel_seed_eval(seed: int, queries: np.ndarray) -> np.ndarray:
    """SeedForPixelSample(seed, x, y, sample) for rows (x, y, sample)."""
    q = np.ascontiguousarray(queries, np.int64).reshape(-1, 3)
    out = np.empty(q.shape[0], np.uint64)
    _lib.check(_lib.lib().yrc_pixel_seed_eval(C.c_uint64(seed), _lib.ptr(q), q.shape[0], _lib.ptr(out)))
    return out
