"""ctypes binding of libyrcuda (include/yrcuda.h).

The library is built in-tree (``python -m yaoray_b200.build``) and loaded from
this package directory. There is no fallback: if the library is missing or
fails to load, every entry point raises ``YrcError`` — the CUDA path is the
only implementation.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libyrcuda.so"

YRC_OK = 0
YRC_ERR_INVALID_ARGUMENT = 1
YRC_ERR_CUDA = 2
YRC_ERR_OUT_OF_MEMORY = 3
YRC_ERR_CANCELLED = 4
YRC_ERR_UNSUPPORTED = 5
YRC_ERR_DEVICE_FAULT = 6
YRC_ERR_BUILD = 7

YRC_TRACE_CLOSEST = 0
YRC_TRACE_ANY = 1
YRC_TRACE_STATS = 2
YRC_PROBE_MAX_HITS = 64
YRC_NOALLOC_STATS_MAX_RAYS = 262144
YRC_NRC_QUERY_FLOATS = 16
YRC_NRC_WEIGHT_COUNT = 6 * 64 * 64
YRC_NRC_GRID_COUNT = 16 * 524288 * 2

STATUS_NAMES = {
    0: "ok",
    1: "invalid argument",
    2: "cuda error",
    3: "out of memory",
    4: "cancelled",
    5: "unsupported",
    6: "device fault",
    7: "build error",
}


class YrcError(RuntimeError):
    """A libyrcuda call failed; ``status`` is the yrc_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


# ---------------------------------------------------------------- structures

class Primitive(C.Structure):
    _fields_ = [("first_index", C.c_uint32), ("index_count", C.c_uint32), ("material_index", C.c_int32),
                ("flags", C.c_uint32)]


class Sphere(C.Structure):
    _fields_ = [("center", C.c_float * 3), ("radius", C.c_float), ("material_index", C.c_int32),
                ("area_light_index", C.c_int32), ("flip_normals", C.c_int32), ("reserved", C.c_int32)]


class InstanceDesc(C.Structure):
    _fields_ = [("primitive", C.c_int32), ("object_to_world", C.c_float * 16)]


class Geometry(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("vertex_count", C.c_int64), ("vertex_stride", C.c_int64),
                ("indices", C.c_void_p), ("index_count", C.c_int64),
                ("primitives", C.c_void_p), ("primitive_count", C.c_int32),
                ("spheres", C.c_void_p), ("sphere_count", C.c_int32),
                ("instances", C.c_void_p), ("instance_count", C.c_int32)]


class BvhOptions(C.Structure):
    _fields_ = [("split_method", C.c_int32), ("max_leaf_triangles", C.c_int32), ("thread_count", C.c_int32),
                ("parallel_min_subtree_size", C.c_int32)]


class BvhView(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("node_count", C.c_int64),
                ("primitive_indices", C.c_void_p), ("primitive_index_count", C.c_int64),
                ("primitives", C.c_void_p), ("primitive_count", C.c_int64),
                ("max_depth", C.c_int32)]


class BlasView(C.Structure):
    _fields_ = [("mesh_primitive", C.c_int32), ("object_bounds_min", C.c_float * 3),
                ("object_bounds_max", C.c_float * 3), ("bvh", BvhView)]


class PreparedInstance(C.Structure):
    _fields_ = [("primitive", C.c_int32), ("blas_index", C.c_int32), ("object_to_world", C.c_float * 16),
                ("world_to_object", C.c_float * 16), ("world_bounds_min", C.c_float * 3),
                ("world_bounds_max", C.c_float * 3)]


class TlasPrimitive(C.Structure):
    _fields_ = [("kind", C.c_int32), ("instance", C.c_int32), ("sphere", C.c_int32),
                ("world_bounds_min", C.c_float * 3), ("world_bounds_max", C.c_float * 3)]


class TwoLevelView(C.Structure):
    _fields_ = [("blases", C.c_void_p), ("blas_count", C.c_int32),
                ("instances", C.c_void_p), ("instance_count", C.c_int32),
                ("tlas_nodes", C.c_void_p), ("tlas_node_count", C.c_int64),
                ("tlas_primitive_indices", C.c_void_p), ("tlas_primitive_index_count", C.c_int64),
                ("tlas_primitives", C.c_void_p), ("tlas_primitive_count", C.c_int64),
                ("tlas_max_depth", C.c_int32)]


class TraceStats(C.Structure):
    _fields_ = [("node_tests", C.c_uint64), ("triangle_tests", C.c_uint64), ("sphere_tests", C.c_uint64),
                ("rays", C.c_uint64)]


# numpy dtypes matching the C structs
NODE_DTYPE = np.dtype([("bounds_min", "<f4", 3), ("bounds_max", "<f4", 3), ("payload_offset", "<i4"),
                       ("primitive_count", "<i4")])
BVH_PRIM_DTYPE = np.dtype([("kind", "<i4"), ("mesh_primitive", "<i4"), ("sphere", "<i4"),
                           ("local_triangle", "<i4"), ("flat_triangle_index", "<i4")])
PRIM_DTYPE = np.dtype([("first_index", "<u4"), ("index_count", "<u4"), ("material_index", "<i4"),
                       ("flags", "<u4")])
SPHERE_DTYPE = np.dtype([("center", "<f4", 3), ("radius", "<f4"), ("material_index", "<i4"),
                         ("area_light_index", "<i4"), ("flip_normals", "<i4"), ("reserved", "<i4")])
INSTANCE_DTYPE = np.dtype([("primitive", "<i4"), ("object_to_world", "<f4", 16)])
PREPARED_INSTANCE_DTYPE = np.dtype([("primitive", "<i4"), ("blas_index", "<i4"), ("object_to_world", "<f4", 16),
                                    ("world_to_object", "<f4", 16), ("world_bounds_min", "<f4", 3),
                                    ("world_bounds_max", "<f4", 3)])
TLAS_PRIM_DTYPE = np.dtype([("kind", "<i4"), ("instance", "<i4"), ("sphere", "<i4"),
                            ("world_bounds_min", "<f4", 3), ("world_bounds_max", "<f4", 3)])
RAY_DTYPE = np.dtype([("origin", "<f4", 3), ("t_min", "<f4"), ("direction", "<f4", 3), ("t_max", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("id", "<i4"), ("u", "<f4"), ("v", "<f4")])

assert NODE_DTYPE.itemsize == 32 and RAY_DTYPE.itemsize == 32 and HIT_DTYPE.itemsize == 16
assert PREPARED_INSTANCE_DTYPE.itemsize == C.sizeof(PreparedInstance)
assert TLAS_PRIM_DTYPE.itemsize == C.sizeof(TlasPrimitive)
assert INSTANCE_DTYPE.itemsize == C.sizeof(InstanceDesc)
assert SPHERE_DTYPE.itemsize == C.sizeof(Sphere)


_LIB = None


def lib() -> C.CDLL:
    """The loaded libyrcuda; raises YrcError when it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise YrcError(YRC_ERR_UNSUPPORTED,
                       f"{LIB_PATH} is not built; run `python -m yaoray_b200.build` (no CPU fallback exists)")
    L = C.CDLL(str(LIB_PATH))
    P, I64, I32 = C.c_void_p, C.c_int64, C.c_int32
    sig = {
        "yrc_last_error": (C.c_char_p, []),
        "yrc_version": (C.c_char_p, []),
        "yrc_device_available": (C.c_int, []),
        "yrc_bvh_options_default": (None, [P]),
        "yrc_bvh_build": (C.c_int, [P, P, P]),
        "yrc_bvh_build_device": (C.c_int, [P, P, P, P]),
        "yrc_two_level_build_device": (C.c_int, [P, P, P, P]),
        "yrc_bvh_get_view": (C.c_int, [P, P]),
        "yrc_bvh_destroy": (None, [P]),
        "yrc_two_level_build": (C.c_int, [P, P, P]),
        "yrc_two_level_get_view": (C.c_int, [P, P]),
        "yrc_two_level_destroy": (None, [P]),
        "yrc_accel_create_flat": (C.c_int, [P, P, P]),
        "yrc_accel_create_two_level": (C.c_int, [P, P, P]),
        "yrc_accel_destroy": (None, [P]),
        "yrc_accel_device_bytes": (I64, [P]),
        "yrc_trace_device": (C.c_int, [P, P, I64, I32, P, P, P, P]),
        "yrc_trace_host": (C.c_int, [P, P, I64, I32, P, P, P, P]),
        "yrc_trace_stats_device": (C.c_int, [P, P, I64, I32, P, P, P, P]),
        "yrc_trace_stats_device_noalloc": (C.c_int, [P, P, I64, I32, P, P, P, P]),
        "yrc_probe_device": (C.c_int, [P, P, P, I64, P, P, P, P, P]),
        "yrc_accel_check": (C.c_int, [P]),
        "yrc_accel_autotune": (C.c_int, [P, P, I64, I32, P, P]),
        "yrc_accel_set_trace_shape": (C.c_int, [P, I32, I32]),
        "yrc_accel_get_trace_shape": (I32, [P, I32]),
        "yrc_accel_autotune_host": (C.c_int, [P, P, I64, I32, P]),
        "yrc_accel_set_host_trace_shape": (C.c_int, [P, I32, I32]),
        "yrc_accel_get_host_trace_shape": (I32, [P, I32]),
        "yrc_accel_set_wide": (C.c_int, [P, I32]),
        "yrc_accel_get_wide": (I32, [P]),
        "yrc_accel_set_ray_order": (C.c_int, [P, I32, I32, C.c_float]),
        "yrc_accel_get_ray_order": (I32, [P]),
        "yrc_accel_set_timing": (C.c_int, [P, I32]),
        "yrc_accel_last_timing": (C.c_int, [P, P, P]),
        "yrc_stream_synchronize": (C.c_int, [P]),
        "yrc_nrc_create": (C.c_int, [P, C.c_float, C.c_uint64, P]),
        "yrc_nrc_destroy": (None, [P]),
        "yrc_nrc_set_params": (C.c_int, [P, P, P]),
        "yrc_nrc_get_params": (C.c_int, [P, P, P]),
        "yrc_nrc_get_averaged_params": (C.c_int, [P, P, P]),
        "yrc_nrc_set_average_decay": (C.c_int, [P, C.c_float]),
        "yrc_nrc_infer": (C.c_int, [P, P, I64, P, P]),
        "yrc_nrc_train_step": (C.c_int, [P, P, P, I64, P, P]),
        "yrc_nrc_gradients": (C.c_int, [P, P, P, I64, P, P, P]),
        "yrc_nrc_check": (C.c_int, [P]),
        "yrc_nrc_copy_state": (C.c_int, [P, P]),
        "yrc_sampler_eval": (C.c_int, [I32, C.c_uint64, I32, P, I64, I32, P]),
        "yrc_rng_eval": (C.c_int, [P, I64, I32, P]),
        "yrc_pixel_seed_eval": (C.c_int, [C.c_uint64, P, I64, P]),
        "yrc_texture_sample_eval": (C.c_int, [P, P, P, I64, P]),
        "yrc_texture_mip_chain_eval": (C.c_int, [P, P, I64, P, P]),
        "yrc_measured_eval": (C.c_int, [P, P, I64, P, P]),
        "yrc_measured_sample": (C.c_int, [P, P, I64, P]),
        "yrc_bsdf_eval": (C.c_int, [P, P, P, I64, P, P]),
        "yrc_bsdf_sample": (C.c_int, [P, P, P, I64, P]),
        "yrc_bssrdf_eval": (C.c_int, [P, P, P, C.c_float, P, P, P, I64, P, P, P]),
        "yrc_bssrdf_pdf_sp": (C.c_int, [P, P, P, C.c_float, P, I64, P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = L
    return L


def check(status: int) -> None:
    """Raises YrcError with the library's message when status != YRC_OK."""
    if status != YRC_OK:
        msg = lib().yrc_last_error().decode(errors="replace")
        raise YrcError(status, msg)


def ptr(a) -> int | None:
    """Address of a contiguous numpy array or torch tensor (None if empty)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data if a.size else None
    return a.data_ptr() if a.numel() else None
