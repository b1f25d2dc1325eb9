"""Acceleration structures and GPU traversal — the Python mirror of the
reference's accel API (include/yaoray/accel/{bvh,two_level_bvh,acceleration}.hpp).

    build_bvh(geometry)            -> RenderBvh      BuildBvh            (bvh_builder.cpp:269-286)
    build_two_level_bvh(geometry)  -> TwoLevelBvh    BuildTwoLevelBvh    (two_level_bvh.cpp:257-331)
    build_render_acceleration(g)   -> RenderBvh | TwoLevelBvh            (acceleration.cpp:28-46)
    DeviceAccelerator(g, accel).intersect(rays)      IntersectBvh / IntersectTwoLevelBvh
    DeviceAccelerator(g, accel).probe(rays, targets) IntersectAccelerationProbe

Builders run on the host (C++, multi-threaded) and produce the reference's
exact layout; traversal runs on the GPU through libyrcuda. Rays are
``(N, 8) float32`` rows ``origin.xyz, t_min, direction.xyz, t_max`` and
closest hits ``(N, 4)`` rows ``t, id (int32 bits), u, v`` where id >= 0 is the
flat triangle index, -1 a miss and <= -2 sphere ``-2 - id``.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, lib, ptr

# Compiled launch shapes of the closest / any-hit traversal kernel
# (YRC_TRACE_SHAPES): the autotuner's candidates.
TRACE_SHAPES = 17


# ------------------------------------------------------------------ geometry

@dataclass
class SceneGeometry:
    """GeometryView (include/yaoray/scene/geometry.hpp:44-71) as numpy arrays."""

    positions: np.ndarray                       # (V, 3) float32
    indices: np.ndarray                         # (I,) uint32
    primitives: np.ndarray                      # PRIM_DTYPE
    spheres: np.ndarray = field(default_factory=lambda: np.zeros(0, _lib.SPHERE_DTYPE))
    instances: np.ndarray = field(default_factory=lambda: np.zeros(0, _lib.INSTANCE_DTYPE))

    def __post_init__(self):
        self.positions = np.ascontiguousarray(self.positions, dtype=np.float32).reshape(-1, 3)
        self.indices = np.ascontiguousarray(self.indices, dtype=np.uint32).reshape(-1)
        self.primitives = np.ascontiguousarray(self.primitives, dtype=_lib.PRIM_DTYPE).reshape(-1)
        self.spheres = np.ascontiguousarray(self.spheres, dtype=_lib.SPHERE_DTYPE).reshape(-1)
        self.instances = np.ascontiguousarray(self.instances, dtype=_lib.INSTANCE_DTYPE).reshape(-1)

    @staticmethod
    def from_meshes(meshes, spheres=None, instances=None) -> "SceneGeometry":
        """Concatenates [(positions (V,3), triangles (T,3))] into one geometry
        with one RenderPrimitive per mesh."""
        pos, idx, prims = [], [], []
        vbase = ibase = 0
        for p, t in meshes:
            p = np.asarray(p, np.float32).reshape(-1, 3)
            t = np.asarray(t, np.uint32).reshape(-1, 3)
            pos.append(p)
            idx.append((t + vbase).reshape(-1))
            prims.append((ibase, t.size, 0, 0))
            vbase += p.shape[0]
            ibase += t.size
        sp = np.zeros(0, _lib.SPHERE_DTYPE)
        if spheres is not None and len(spheres):
            s = np.asarray(spheres, np.float32).reshape(-1, 4)
            sp = np.zeros(s.shape[0], _lib.SPHERE_DTYPE)
            sp["center"] = s[:, :3]
            sp["radius"] = s[:, 3]
            sp["area_light_index"] = -1
        inst = np.zeros(0, _lib.INSTANCE_DTYPE)
        if instances is not None and len(instances):
            inst = np.zeros(len(instances), _lib.INSTANCE_DTYPE)
            for k, (prim, m) in enumerate(instances):
                inst[k]["primitive"] = prim
                inst[k]["object_to_world"] = np.asarray(m, np.float32).reshape(16)
        return SceneGeometry(
            np.concatenate(pos) if pos else np.zeros((0, 3), np.float32),
            np.concatenate(idx) if idx else np.zeros(0, np.uint32),
            np.array(prims, dtype=_lib.PRIM_DTYPE) if prims else np.zeros(0, _lib.PRIM_DTYPE),
            sp, inst)

    @property
    def triangle_count(self) -> int:
        return int(self.primitives["index_count"].sum() // 3) if self.primitives.size else 0

    def c_struct(self) -> _lib.Geometry:
        g = _lib.Geometry()
        g.positions = ptr(self.positions)
        g.vertex_count = self.positions.shape[0]
        g.vertex_stride = 12
        g.indices = ptr(self.indices)
        g.index_count = self.indices.size
        g.primitives = ptr(self.primitives)
        g.primitive_count = self.primitives.size
        g.spheres = ptr(self.spheres)
        g.sphere_count = self.spheres.size
        g.instances = ptr(self.instances)
        g.instance_count = self.instances.size
        return g


# ------------------------------------------------------------------ BVHs

@dataclass
class RenderBvh:
    """RenderBvh (include/yaoray/accel/bvh.hpp:72-81); binary nodes only."""

    nodes: np.ndarray              # NODE_DTYPE (32 B each)
    primitive_indices: np.ndarray  # int32
    primitives: np.ndarray         # BVH_PRIM_DTYPE
    max_depth: int = 0

    @property
    def total_triangles(self) -> int:
        return int((self.primitives["kind"] == 0).sum())

    @property
    def total_spheres(self) -> int:
        return int((self.primitives["kind"] != 0).sum())

    def view(self) -> _lib.BvhView:
        v = _lib.BvhView()
        self.nodes = np.ascontiguousarray(self.nodes, _lib.NODE_DTYPE)
        self.primitive_indices = np.ascontiguousarray(self.primitive_indices, np.int32)
        self.primitives = np.ascontiguousarray(self.primitives, _lib.BVH_PRIM_DTYPE)
        v.nodes = ptr(self.nodes)
        v.node_count = self.nodes.size
        v.primitive_indices = ptr(self.primitive_indices)
        v.primitive_index_count = self.primitive_indices.size
        v.primitives = ptr(self.primitives)
        v.primitive_count = self.primitives.size
        v.max_depth = self.max_depth
        return v


@dataclass
class TwoLevelBvh:
    """TwoLevelBvh (include/yaoray/accel/two_level_bvh.hpp:42-46)."""

    blases: list                   # [(mesh_primitive, object_bounds (2,3), RenderBvh)]
    instances: np.ndarray          # PREPARED_INSTANCE_DTYPE
    tlas: RenderBvh                # nodes / primitive_indices / max_depth (primitives unused)
    tlas_primitives: np.ndarray    # TLAS_PRIM_DTYPE

    def view(self):
        blas_arr = (_lib.BlasView * max(len(self.blases), 1))()
        keep = []
        for k, (mp, bounds, bvh) in enumerate(self.blases):
            blas_arr[k].mesh_primitive = mp
            for a in range(3):
                blas_arr[k].object_bounds_min[a] = float(bounds[0][a])
                blas_arr[k].object_bounds_max[a] = float(bounds[1][a])
            blas_arr[k].bvh = bvh.view()
            keep.append(bvh)
        self.instances = np.ascontiguousarray(self.instances, _lib.PREPARED_INSTANCE_DTYPE)
        self.tlas_primitives = np.ascontiguousarray(self.tlas_primitives, _lib.TLAS_PRIM_DTYPE)
        tv = self.tlas.view()
        v = _lib.TwoLevelView()
        v.blases = C.addressof(blas_arr)
        v.blas_count = len(self.blases)
        v.instances = ptr(self.instances)
        v.instance_count = self.instances.size
        v.tlas_nodes = tv.nodes
        v.tlas_node_count = tv.node_count
        v.tlas_primitive_indices = tv.primitive_indices
        v.tlas_primitive_index_count = tv.primitive_index_count
        v.tlas_primitives = ptr(self.tlas_primitives)
        v.tlas_primitive_count = self.tlas_primitives.size
        v.tlas_max_depth = self.tlas.max_depth
        return v, (blas_arr, keep)


def _options(split_method: str, max_leaf_triangles: int, thread_count: int,
             parallel_min_subtree_size: int) -> _lib.BvhOptions:
    o = _lib.BvhOptions()
    o.split_method = {"sah": 0, "median": 1}[split_method]
    o.max_leaf_triangles = max_leaf_triangles
    o.thread_count = thread_count
    o.parallel_min_subtree_size = parallel_min_subtree_size
    return o


def _copy_bvh(v: _lib.BvhView) -> RenderBvh:
    def arr(p, n, dt):
        if n == 0 or not p:
            return np.zeros(0, dt)
        buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(p)
        return np.frombuffer(buf, dtype=dt, count=n).copy()
    return RenderBvh(arr(v.nodes, v.node_count, _lib.NODE_DTYPE),
                     arr(v.primitive_indices, v.primitive_index_count, np.int32),
                     arr(v.primitives, v.primitive_count, _lib.BVH_PRIM_DTYPE), int(v.max_depth))


def build_bvh(geometry: SceneGeometry, split_method: str = "sah", max_leaf_triangles: int = 4,
              thread_count: int = 0, parallel_min_subtree_size: int = 1024) -> RenderBvh:
    """BuildBvh: the reference's binned-SAH (or median) BVH, byte-identical."""
    L = lib()
    g = geometry.c_struct()
    o = _options(split_method, max_leaf_triangles, thread_count, parallel_min_subtree_size)
    h = C.c_void_p()
    check(L.yrc_bvh_build(C.byref(g), C.byref(o), C.byref(h)))
    try:
        v = _lib.BvhView()
        check(L.yrc_bvh_get_view(h, C.byref(v)))
        return _copy_bvh(v)
    finally:
        L.yrc_bvh_destroy(h)


def build_bvh_device(geometry: SceneGeometry, split_method: str = "sah", max_leaf_triangles: int = 4):
    """BuildBvh with the hierarchy built on the current CUDA device (byte-identical
    to build_bvh). Returns (bvh, built_on_device): ranges the reference splits
    at the median (std::nth_element) make the host builder build it."""
    L = lib()
    g = geometry.c_struct()
    o = _options(split_method, max_leaf_triangles, 0, 1024)
    h = C.c_void_p()
    flag = C.c_int32(0)
    check(L.yrc_bvh_build_device(C.byref(g), C.byref(o), C.byref(h), C.byref(flag)))
    try:
        v = _lib.BvhView()
        check(L.yrc_bvh_get_view(h, C.byref(v)))
        return _copy_bvh(v), bool(flag.value)
    finally:
        L.yrc_bvh_destroy(h)


def build_two_level_bvh(geometry: SceneGeometry, split_method: str = "sah", max_leaf_triangles: int = 4,
                        thread_count: int = 0, parallel_min_subtree_size: int = 1024,
                        device: bool = False) -> TwoLevelBvh:
    """BuildTwoLevelBvh: one BLAS per mesh primitive + TLAS over instances;
    with `device` the BLASes are built on the current CUDA device
    (byte-identical)."""
    L = lib()
    g = geometry.c_struct()
    o = _options(split_method, max_leaf_triangles, thread_count, parallel_min_subtree_size)
    h = C.c_void_p()
    if device:
        check(L.yrc_two_level_build_device(C.byref(g), C.byref(o), C.byref(h), None))
    else:
        check(L.yrc_two_level_build(C.byref(g), C.byref(o), C.byref(h)))
    try:
        v = _lib.TwoLevelView()
        check(L.yrc_two_level_get_view(h, C.byref(v)))
        blases = []
        for k in range(v.blas_count):
            b = _lib.BlasView.from_address(v.blases + k * C.sizeof(_lib.BlasView))
            bounds = np.array([list(b.object_bounds_min), list(b.object_bounds_max)], np.float32)
            blases.append((int(b.mesh_primitive), bounds, _copy_bvh(b.bvh)))
        def arr(p, n, dt):
            if n == 0 or not p:
                return np.zeros(0, dt)
            buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(p)
            return np.frombuffer(buf, dtype=dt, count=n).copy()
        tlas = RenderBvh(arr(v.tlas_nodes, v.tlas_node_count, _lib.NODE_DTYPE),
                         arr(v.tlas_primitive_indices, v.tlas_primitive_index_count, np.int32),
                         np.zeros(0, _lib.BVH_PRIM_DTYPE), int(v.tlas_max_depth))
        return TwoLevelBvh(blases, arr(v.instances, v.instance_count, _lib.PREPARED_INSTANCE_DTYPE), tlas,
                           arr(v.tlas_primitives, v.tlas_primitive_count, _lib.TLAS_PRIM_DTYPE))
    finally:
        L.yrc_two_level_destroy(h)


def build_render_acceleration(geometry: SceneGeometry, **options):
    """BuildRenderAcceleration: explicit instances select the two-level path."""
    if geometry.instances.size:
        return build_two_level_bvh(geometry, **options)
    return build_bvh(geometry, **options)


# --------------------------------------------------------------- device side

def _torch():
    import torch
    return torch


def _stream_handle(stream) -> int | None:
    if stream is None:
        torch = _torch()
        return torch.cuda.current_stream().cuda_stream
    return stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)


class DeviceAccelerator:
    """Geometry + BVH resident in HBM in the traversal layout (libyrcuda)."""

    def __init__(self, geometry: SceneGeometry, accel):
        L = lib()
        self._handle = C.c_void_p()
        g = geometry.c_struct()
        if isinstance(accel, TwoLevelBvh):
            v, keep = accel.view()
            check(L.yrc_accel_create_two_level(C.byref(g), C.byref(v), C.byref(self._handle)))
            del keep
            self.two_level = True
        else:
            v = accel.view()
            check(L.yrc_accel_create_flat(C.byref(g), C.byref(v), C.byref(self._handle)))
            self.two_level = False

    def close(self):
        if getattr(self, "_handle", None) and self._handle.value:
            lib().yrc_accel_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(lib().yrc_accel_device_bytes(self._handle))

    def autotune(self, rays, any_hit: bool = False, stream=None) -> dict:
        """Times every launch shape on `rays` (CUDA tensor) and keeps the
        fastest; returns {shape: milliseconds} and the chosen shape."""
        times = (C.c_float * TRACE_SHAPES)()
        n = rays.numel() // 8
        check(lib().yrc_accel_autotune(self._handle, ptr(rays), n, _lib.YRC_TRACE_ANY if any_hit else 0,
                                       _stream_handle(stream), times))
        return {"times_ms": [round(float(t), 4) for t in times],
                "shape": int(lib().yrc_accel_get_trace_shape(self._handle, int(any_hit)))}

    def set_trace_shape(self, shape: int, any_hit: bool = False) -> None:
        check(lib().yrc_accel_set_trace_shape(self._handle, int(any_hit), shape))

    def autotune_host(self, rays: np.ndarray, any_hit: bool = False) -> dict:
        """Times yrc_trace_host on host rays (N, 8) float32 (pinned memory,
        like the caller's) per launch shape and keeps the fastest for the
        host path; returns {shape: milliseconds per call} and the choice."""
        times = (C.c_float * TRACE_SHAPES)()
        n = rays.size // 8
        check(lib().yrc_accel_autotune_host(self._handle, ptr(rays), n, _lib.YRC_TRACE_ANY if any_hit else 0, times))
        return {"times_ms": [round(float(t), 3) for t in times],
                "shape": int(lib().yrc_accel_get_host_trace_shape(self._handle, int(any_hit)))}

    def set_host_trace_shape(self, shape: int, any_hit: bool = False) -> None:
        """Launch shape of the host-buffer path (-1: follow set_trace_shape)."""
        check(lib().yrc_accel_set_host_trace_shape(self._handle, int(any_hit), shape))

    @property
    def wide(self) -> bool:
        """True while closest / any-hit traces use the four-wide copy of the
        hierarchy (flat, triangle-only BVHs; same hits as the binary one)."""
        return bool(lib().yrc_accel_get_wide(self._handle))

    def set_wide(self, enable: bool) -> None:
        check(lib().yrc_accel_set_wide(self._handle, int(enable)))

    RAY_ORDER_MODES = {"off": 0, "direction": 1, "two-point": 2}

    @property
    def ray_order(self) -> str:
        """Reordering applied before device traces: "off", "direction" (key:
        origin and direction) or "two-point" (key: origin and a point along
        the ray)."""
        mode = int(lib().yrc_accel_get_ray_order(self._handle))
        return {v: k for k, v in self.RAY_ORDER_MODES.items()}[mode]

    def set_ray_order(self, mode: str, key_bits: int = 0, length: float = 0.05) -> None:
        check(lib().yrc_accel_set_ray_order(self._handle, self.RAY_ORDER_MODES[mode], key_bits, length))

    def set_timing(self, enable: bool) -> None:
        """Records CUDA events around each device trace's reordering and
        traversal kernel (read back with last_timing)."""
        check(lib().yrc_accel_set_timing(self._handle, int(enable)))

    def last_timing(self) -> tuple[float, float]:
        """(reordering ms, traversal kernel ms) of the last device trace."""
        order_ms, trace_ms = C.c_float(), C.c_float()
        check(lib().yrc_accel_last_timing(self._handle, C.byref(order_ms), C.byref(trace_ms)))
        return float(order_ms.value), float(trace_ms.value)

    def check(self) -> None:
        """Synchronises and raises if a kernel recorded an error status."""
        check(lib().yrc_accel_check(self._handle))

    # -- device-resident rays (torch CUDA tensors) --------------------------
    def intersect(self, rays, any_hit: bool = False, hits=None, occluded=None, instances=None, stream=None):
        """Traces (N, 8) float32 CUDA rays; returns hits (N, 4) float32 (id as
        int32 bits) or occluded (N,) uint8. Asynchronous on `stream`."""
        torch = _torch()
        assert rays.is_cuda and rays.dtype == torch.float32 and rays.is_contiguous()
        n = rays.numel() // 8
        if any_hit:
            if occluded is None:
                occluded = torch.empty(n, dtype=torch.uint8, device=rays.device)
            check(lib().yrc_trace_device(self._handle, ptr(rays), n, _lib.YRC_TRACE_ANY, None, None,
                                         ptr(occluded), _stream_handle(stream)))
            return occluded
        if hits is None:
            hits = torch.empty((n, 4), dtype=torch.float32, device=rays.device)
        check(lib().yrc_trace_device(self._handle, ptr(rays), n, _lib.YRC_TRACE_CLOSEST, ptr(hits),
                                     ptr(instances), None, _stream_handle(stream)))
        return hits

    def trace_stats(self, rays, any_hit: bool = False, stream=None):
        """Per-ray BvhTraceStats (node, triangle, sphere tests) as uint32 tensors."""
        torch = _torch()
        n = rays.numel() // 8
        out = torch.empty((3, n), dtype=torch.int32, device=rays.device)
        flags = _lib.YRC_TRACE_ANY if any_hit else _lib.YRC_TRACE_CLOSEST
        check(lib().yrc_trace_stats_device(self._handle, ptr(rays), n, flags, ptr(out[0]), ptr(out[1]),
                                           ptr(out[2]), _stream_handle(stream)))
        return out

    def probe(self, rays, targets, stream=None):
        """IntersectAccelerationProbe; targets (N, 4) int32 rows (primitive,
        instance, sphere, 0). Returns (hits (N, 64, 4), instances (N, 64),
        counts (N,), exhausted (N,))."""
        torch = _torch()
        n = rays.numel() // 8
        dev = rays.device
        hits = torch.zeros((n, _lib.YRC_PROBE_MAX_HITS, 4), dtype=torch.float32, device=dev)
        inst = torch.full((n, _lib.YRC_PROBE_MAX_HITS), -1, dtype=torch.int32, device=dev)
        counts = torch.empty(n, dtype=torch.int32, device=dev)
        exhausted = torch.empty(n, dtype=torch.uint8, device=dev)
        check(lib().yrc_probe_device(self._handle, ptr(rays), ptr(targets), n, ptr(hits), ptr(inst), ptr(counts),
                                     ptr(exhausted), _stream_handle(stream)))
        return hits, inst, counts, exhausted

    # -- host-resident rays (the drop-in C-ABI path) -------------------------
    def intersect_host(self, rays: np.ndarray, any_hit: bool = False, with_stats: bool = False,
                       out=None, instances_out=None):
        """Traces host rays (N, 8) float32 through yrc_trace_host (copies in,
        traces, copies out). Returns hits (N, 4) float32 or occluded (N,)
        uint8, plus a stats dict when with_stats."""
        n = rays.size // 8
        flags = (_lib.YRC_TRACE_ANY if any_hit else 0) | (_lib.YRC_TRACE_STATS if with_stats else 0)
        stats = _lib.TraceStats()
        if any_hit:
            out = np.empty(n, np.uint8) if out is None else out
            check(lib().yrc_trace_host(self._handle, ptr(rays), n, flags, None, None, ptr(out),
                                       C.byref(stats) if with_stats else None))
        else:
            out = np.empty((n, 4), np.float32) if out is None else out
            check(lib().yrc_trace_host(self._handle, ptr(rays), n, flags, ptr(out), ptr(instances_out), None,
                                       C.byref(stats) if with_stats else None))
        if with_stats:
            return out, {"node_tests": stats.node_tests, "triangle_tests": stats.triangle_tests,
                         "sphere_tests": stats.sphere_tests, "rays": stats.rays}
        return out


def hit_ids(hits) -> np.ndarray:
    """The int32 id column of a (N, 4) float32 hit array (numpy or torch)."""
    if not isinstance(hits, np.ndarray):
        hits = hits.detach().cpu().numpy()
    return np.ascontiguousarray(hits[..., 1]).view(np.int32)
