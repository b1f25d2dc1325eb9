"""Neural radiance cache (libyrcuda's yrc_nrc_*): hash-grid + spherical
harmonics encoding into a 64-wide MLP evaluated and trained on the tensor
cores. Queries are (N, 16) float32 CUDA tensors — position[3], roughness,
direction[3], normal[3], diffuse albedo[3], specular albedo[3]; radiance
targets and outputs are (N, 4) float32 (RGB, w unused).

The reference renderer has no radiance cache; this is an addition of this
backend, used by the path tracer to terminate paths early.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib, ptr
from .accel import _stream_handle, _torch

LEVELS, TABLE, WIDTH = 16, 1 << 19, 64


class RadianceCache:
    def __init__(self, box_lo, box_extent: float, seed: int = 0):
        lo = (C.c_float * 3)(*[float(v) for v in box_lo])
        self._handle = C.c_void_p()
        check(lib().yrc_nrc_create(lo, float(box_extent), int(seed), C.byref(self._handle)))
        self.box_lo = tuple(float(v) for v in box_lo)
        self.box_extent = float(box_extent)

    def close(self):
        if getattr(self, "_handle", None):
            lib().yrc_nrc_destroy(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def copy_from(self, other: "RadianceCache") -> None:
        """Makes this cache an exact copy of `other` (parameters, optimiser
        state, moving average), e.g. to evaluate one trained state several
        times."""
        check(lib().yrc_nrc_copy_state(self._handle, other._handle))

    def set_params(self, weights: np.ndarray | None = None, grid: np.ndarray | None = None) -> None:
        """weights (6, 64, 64) and grid (16, 2^19, 2) float32 master values."""
        w = None if weights is None else np.ascontiguousarray(weights, np.float32)
        g = None if grid is None else np.ascontiguousarray(grid, np.float32)
        if w is not None:
            assert w.size == _lib.YRC_NRC_WEIGHT_COUNT
        if g is not None:
            assert g.size == _lib.YRC_NRC_GRID_COUNT
        check(lib().yrc_nrc_set_params(self._handle, ptr(w), ptr(g)))

    def get_params(self):
        w = np.empty((6, WIDTH, WIDTH), np.float32)
        g = np.empty((LEVELS, TABLE, 2), np.float32)
        check(lib().yrc_nrc_get_params(self._handle, ptr(w), ptr(g)))
        return w, g

    def set_average_decay(self, decay: float) -> None:
        """Largest decay of the parameter moving average (default 0.99); set
        it before attaching the cache to a scene."""
        check(lib().yrc_nrc_set_average_decay(self._handle, float(decay)))

    def get_averaged_params(self):
        """The moving average of the parameters (decay min(0.99, (1+t)/(10+t))
        at optimiser step t), which a render may query instead."""
        w = np.empty((6, WIDTH, WIDTH), np.float32)
        g = np.empty((LEVELS, TABLE, 2), np.float32)
        check(lib().yrc_nrc_get_averaged_params(self._handle, ptr(w), ptr(g)))
        return w, g

    def infer(self, queries, out=None, stream=None):
        torch = _torch()
        n = queries.shape[0]
        assert queries.is_cuda and queries.dtype == torch.float32 and queries.shape[1] == 16
        if out is None:
            out = torch.empty((n, 4), dtype=torch.float32, device=queries.device)
        check(lib().yrc_nrc_infer(self._handle, ptr(queries), n, ptr(out), _stream_handle(stream)))
        return out

    def train_step(self, queries, targets, loss_out=None, stream=None) -> None:
        n = queries.shape[0]
        check(lib().yrc_nrc_train_step(self._handle, ptr(queries), ptr(targets), n, ptr(loss_out),
                                       _stream_handle(stream)))

    def gradients(self, queries, targets):
        """(weight gradients (6, 64, 64), grid gradients (16, 2^19, 2), mean loss)."""
        n = queries.shape[0]
        wg = np.empty((6, WIDTH, WIDTH), np.float32)
        gg = np.empty((LEVELS, TABLE, 2), np.float32)
        loss = C.c_float()
        check(lib().yrc_nrc_gradients(self._handle, ptr(queries), ptr(targets), n, ptr(wg), ptr(gg),
                                      C.byref(loss)))
        return wg, gg, float(loss.value)

    def check(self) -> None:
        check(lib().yrc_nrc_check(self._handle))
