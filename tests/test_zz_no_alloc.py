"""yrc_trace_stats_device_noalloc, the stats traversal for callers that cannot
allocate device memory (an application that gives all GPU memory to its own
pool at start-up, or a frame loop that must never enter the CUDA allocator).

Both it and yrc_trace_stats_device are called through the C ABI on the same
rays; its per-ray counters must equal the allocating entry point's bit for bit
(integer counts, no tolerance) on two calls in a row, since consecutive calls
reuse one fixed scratch array that keeps the previous call's contents. Batches
larger than that array are refused before any work is queued.

This file is named to be collected last."""
import ctypes as C

import numpy as np
import pytest

from yaoray_b200 import _lib, accel, scenes
from yaoray_b200.accel import RenderBvh, SceneGeometry

pytestmark = pytest.mark.gpu
MAX_RAYS = _lib.YRC_NOALLOC_STATS_MAX_RAYS


def _stream():
    import torch

    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _counts(fn, handle, rays, n, flags, sentinel):
    """Runs one stats entry point and returns its (3, n) counters; the output
    starts filled with `sentinel` so that unwritten entries show."""
    import torch

    out = torch.full((3, n), sentinel, dtype=torch.int32, device=rays.device)
    status = fn(handle, _lib.ptr(rays), n, flags, _lib.ptr(out[0]), _lib.ptr(out[1]), _lib.ptr(out[2]), _stream())
    assert status == _lib.YRC_OK, _lib.lib().yrc_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def _compare_two_calls(handle, rays, n, flags):
    L = _lib.lib()
    want = _counts(L.yrc_trace_stats_device, handle, rays, n, flags, -1)
    assert (want >= 0).all() and want[0].sum() > 0
    for sentinel in (-1, 0x5A5A5A5A):  # two calls in a row on the shared scratch
        got = _counts(L.yrc_trace_stats_device_noalloc, handle, rays, n, flags, sentinel)
        assert np.array_equal(got, want)
    assert L.yrc_accel_check(handle) == _lib.YRC_OK


@pytest.fixture(scope="module")
def mesh_scene(cuda):
    import torch

    geom = scenes.traversal_scene(seed=7, spheres=64)
    dev = accel.DeviceAccelerator(geom, accel.build_bvh(geom))
    rays = torch.from_numpy(scenes.incoherent_rays(MAX_RAYS + 1, seed=11)).to(cuda)
    return dev, rays


@pytest.mark.parametrize("flags", [_lib.YRC_TRACE_CLOSEST, _lib.YRC_TRACE_ANY])
def test_noalloc_matches_allocating_stats_at_the_maximum(mesh_scene, flags):
    dev, rays = mesh_scene
    _compare_two_calls(dev._handle, rays, MAX_RAYS, flags)


def test_noalloc_matches_on_spheres_and_reference_counts(cuda):
    import torch
    from pathlib import Path

    f = dict(np.load(Path(__file__).resolve().parent / "golden" / "trace_spheres.npz"))
    g = SceneGeometry(f["positions"], f["indices"], f["primitives"], f["spheres"], f["instances"])
    b = RenderBvh(f["bvh_nodes"], f["bvh_primitive_indices"], f["bvh_primitives"], int(f["bvh_max_depth"]))
    dev = accel.DeviceAccelerator(g, b)
    rays = torch.from_numpy(np.ascontiguousarray(f["rays"])).to(cuda)
    n = rays.shape[0]
    _compare_two_calls(dev._handle, rays, n, _lib.YRC_TRACE_CLOSEST)
    got = _counts(_lib.lib().yrc_trace_stats_device_noalloc, dev._handle, rays, n, _lib.YRC_TRACE_CLOSEST, -1)
    for row, key in enumerate(("out_node_tests", "out_triangle_tests", "out_sphere_tests")):
        assert np.array_equal(got[row].astype(np.uint32), f[key]), key


def test_noalloc_refuses_batches_beyond_its_scratch(mesh_scene):
    import torch

    dev, rays = mesh_scene  # holds MAX_RAYS + 1 rays, so even a missed check reads in bounds
    out = torch.full((3, MAX_RAYS + 1), -1, dtype=torch.int32, device=rays.device)
    L = _lib.lib()
    status = L.yrc_trace_stats_device_noalloc(dev._handle, _lib.ptr(rays), MAX_RAYS + 1, _lib.YRC_TRACE_CLOSEST,
                                              _lib.ptr(out[0]), _lib.ptr(out[1]), _lib.ptr(out[2]), _stream())
    assert status == _lib.YRC_ERR_INVALID_ARGUMENT
    assert "fixed maximum of 262144" in L.yrc_last_error().decode()
    torch.cuda.synchronize()
    assert (out == -1).all()  # nothing was queued
