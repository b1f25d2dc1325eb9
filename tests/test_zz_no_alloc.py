"""yrc_trace_stats_device_noalloc, the stats traversal for callers that cannot
allocate device memory (an application that gives all GPU memory to its own
pool at start-up, or a frame loop that must never enter the CUDA allocator).

Both it and yrc_trace_stats_device are called through the C ABI on the same
rays; its per-ray counters must equal the allocating entry point's bit for bit
(integer counts, no tolerance) on two calls in a row, since consecutive calls
reuse one fixed scratch array that keeps the previous call's contents. Batches
larger than that array are refused before any work is queued.

It also checks the property itself: after the accelerator is created, free
device memory and the stream-ordered pool's usage stay the same across
no-allocation calls (the first one included), while the allocating entry point
does show up in the pool's high-water mark, so the check can see an allocation.

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


# CUmemPool_attribute values (cuda.h): pool usage as the driver counts it.
_USED_MEM_CURRENT, _USED_MEM_HIGH = 7, 8


def _default_pool():
    """The current device's default stream-ordered memory pool, through the
    driver API (libyrcuda links its own CUDA runtime, so torch's allocator
    statistics would not see its allocations)."""
    import torch

    cu = C.CDLL("libcuda.so.1")
    dev = C.c_int()
    assert cu.cuDeviceGet(C.byref(dev), torch.cuda.current_device()) == 0
    pool = C.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(C.byref(pool), dev) == 0
    return cu, pool


def _pool_attr(cu, pool, attr):
    v = C.c_uint64()
    assert cu.cuMemPoolGetAttribute(pool, attr, C.byref(v)) == 0
    return v.value


def test_noalloc_calls_take_no_device_memory(cuda):
    import torch

    geom = scenes.traversal_scene(seed=3, spheres=16)
    dev = accel.DeviceAccelerator(geom, accel.build_bvh(geom))
    n = 65536
    rays = torch.from_numpy(scenes.incoherent_rays(n, seed=4)).to(cuda)
    out = torch.full((3, n), -1, dtype=torch.int32, device=cuda)
    L = _lib.lib()
    torch.cuda.synchronize()
    cu, pool = _default_pool()
    zero = C.c_uint64(0)
    assert cu.cuMemPoolSetAttribute(pool, _USED_MEM_HIGH, C.byref(zero)) == 0  # restart the high-water mark
    used0 = _pool_attr(cu, pool, _USED_MEM_CURRENT)
    free0 = torch.cuda.mem_get_info()[0]
    for flags in (_lib.YRC_TRACE_CLOSEST, _lib.YRC_TRACE_ANY, _lib.YRC_TRACE_CLOSEST):
        status = L.yrc_trace_stats_device_noalloc(dev._handle, _lib.ptr(rays), n, flags, _lib.ptr(out[0]),
                                                  _lib.ptr(out[1]), _lib.ptr(out[2]), _stream())
        assert status == _lib.YRC_OK, L.yrc_last_error().decode()
        torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert _pool_attr(cu, pool, _USED_MEM_HIGH) <= used0
    assert (out[0] > 0).any()
    # control: the allocating entry point takes its scratch from that pool
    status = L.yrc_trace_stats_device(dev._handle, _lib.ptr(rays), n, _lib.YRC_TRACE_CLOSEST, _lib.ptr(out[0]),
                                      _lib.ptr(out[1]), _lib.ptr(out[2]), _stream())
    assert status == _lib.YRC_OK
    torch.cuda.synchronize()
    assert _pool_attr(cu, pool, _USED_MEM_HIGH) >= used0 + 16 * n


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
