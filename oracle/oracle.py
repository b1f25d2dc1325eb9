"""TEST ORACLE — Python access to (1) the C restatement of the reference's hot
path (oracle/liboracle.so, built from yr_oracle.c) and (2) the reference
implementation itself (oracle/_ref/libyaoray_ref.so, compiled from the
reference sources by oracle/Makefile, with ref_shim.cpp as its C shim).

Only the tests, ``__graft_entry__.smoke()`` and the benchmark's CPU-baseline
leg use this module, and only as the checker / the timed CPU reference. The
product (yaoray_b200, libyrcuda) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libyaoray_ref.so"
# The reference checkout: $YAORAY_REFERENCE, else "reference" beside the repository root.
REFERENCE_SRC = Path(os.environ.get("YAORAY_REFERENCE", str(HERE.parent.parent / "reference")))

P, I64, I32, U64 = C.c_void_p, C.c_int64, C.c_int32, C.c_uint64


def build(reference: bool = True) -> None:
    """Builds liboracle.so and, when the reference sources are present, _ref."""
    subprocess.run(["make", "-s", "-C", str(HERE), "oracle"], check=True)
    if reference and REFERENCE_SRC.exists():
        jobs = str(min(16, os.cpu_count() or 4))
        subprocess.run(["make", "-s", "-C", str(HERE), f"-j{jobs}", "ref", f"REF={REFERENCE_SRC}"], check=True)
        # the drop-in driver links the product library, built before this step
        subprocess.run(["make", "-s", "-C", str(HERE), f"-j{jobs}", "dropin", f"REF={REFERENCE_SRC}"], check=True)


def ref_available() -> bool:
    return REF_SO.exists()


# --------------------------------------------------------- C restatement

class YoGeometry(C.Structure):
    _fields_ = [("positions", P), ("vertex_count", I64), ("vertex_stride", I64), ("indices", P),
                ("index_count", I64), ("prim_first_count", P), ("primitive_count", I32), ("spheres", P),
                ("sphere_count", I32)]


class YoBvh(C.Structure):
    _fields_ = [("nodes", P), ("node_count", I64), ("primitive_indices", P), ("primitive_index_count", I64),
                ("primitives", P), ("primitive_count", I64)]


class YoTwoLevel(C.Structure):
    _fields_ = [("blases", P), ("blas_count", I32), ("instance_blas", P), ("instance_w2o", P),
                ("instance_count", I32), ("tlas_nodes", P), ("tlas_node_count", I64),
                ("tlas_primitive_indices", P), ("tlas_primitive_index_count", I64), ("tlas_primitives", P),
                ("tlas_primitive_count", I64)]


YO_HIT_DTYPE = np.dtype([("hit", "<i4"), ("t", "<f4"), ("triangle_index", "<i4"), ("mesh_primitive", "<i4"),
                         ("instance", "<i4"), ("sphere", "<i4"), ("u", "<f4"), ("v", "<f4")])


def _p(a):
    return None if a is None or a.size == 0 else a.ctypes.data


_ORACLE = None


def oracle_lib() -> C.CDLL:
    global _ORACLE
    if _ORACLE is None:
        if not ORACLE_SO.exists():
            build(reference=False)
        L = C.CDLL(str(ORACLE_SO))
        L.yo_trace_flat.argtypes = [P, P, P, I64, P, P, P, P, C.c_int]
        L.yo_trace_two_level.argtypes = [P, P, P, I64, P, P, P, P, C.c_int]
        L.yo_probe.argtypes = [P, P, P, P, I64, P, P, P, P]
        L.yo_sampler.argtypes = [C.c_int, U64, C.c_int, P, I64, C.c_int, P]
        L.yo_seed_for_pixel_sample.argtypes = [U64, C.c_int, C.c_int, C.c_int]
        L.yo_seed_for_pixel_sample.restype = U64
        L.yo_rng_floats.argtypes = [U64, C.c_int, P]
        L.yo_texture_sample.argtypes = [C.c_int, C.c_int, P, C.c_int, C.c_int, C.c_int, P, P, I64, P]
        L.yo_texture_mip_chain.argtypes = [C.c_int, C.c_int, P, C.c_int, C.c_int, P, P]
        L.yo_texture_mip_chain.restype = C.c_int
        L.yo_camera_rays.argtypes = [P, C.c_int, C.c_int, P, P, I64, P]
        L.yo_film_accumulate.argtypes = [C.c_int, C.c_int, P, I64, P]
        L.yo_film_accumulate.restype = U64
        _ORACLE = L
    return _ORACLE


class OracleScene:
    """Geometry + BVH arrays held for the C restatement."""

    def __init__(self, geometry, accel):
        self.g_pos = np.ascontiguousarray(geometry.positions, np.float32)
        self.g_idx = np.ascontiguousarray(geometry.indices, np.uint32)
        self.g_prims = np.ascontiguousarray(
            np.stack([geometry.primitives["first_index"], geometry.primitives["index_count"]], 1)
            if geometry.primitives.size else np.zeros((0, 2)), np.uint32)
        sp = geometry.spheres
        self.g_sph = np.ascontiguousarray(
            np.concatenate([sp["center"], sp["radius"][:, None]], 1) if sp.size else np.zeros((0, 4)), np.float32)
        self.geo = YoGeometry(_p(self.g_pos), self.g_pos.shape[0], 12, _p(self.g_idx), self.g_idx.size,
                              _p(self.g_prims), self.g_prims.shape[0], _p(self.g_sph), self.g_sph.shape[0])
        self._keep = []
        self.two_level = hasattr(accel, "blases")
        if self.two_level:
            blases = (YoBvh * max(len(accel.blases), 1))()
            for k, (_, _, b) in enumerate(accel.blases):
                blases[k] = self._bvh(b)
            self._keep.append(blases)
            inst = accel.instances
            self.i_blas = np.ascontiguousarray(inst["blas_index"], np.int32)
            self.i_w2o = np.ascontiguousarray(inst["world_to_object"].reshape(-1, 16), np.float32)
            tp = accel.tlas_primitives
            self.t_prims = np.ascontiguousarray(
                np.stack([tp["kind"], tp["instance"], tp["sphere"]], 1) if tp.size else np.zeros((0, 3)), np.int32)
            t = accel.tlas
            self.t_nodes = np.ascontiguousarray(t.nodes)
            self.t_pi = np.ascontiguousarray(t.primitive_indices, np.int32)
            self.tl = YoTwoLevel(C.addressof(blases), len(accel.blases), _p(self.i_blas), _p(self.i_w2o),
                                 self.i_blas.size, _p(self.t_nodes), self.t_nodes.size, _p(self.t_pi), self.t_pi.size,
                                 _p(self.t_prims), self.t_prims.shape[0])
        else:
            self.bvh = self._bvh(accel)

    def _bvh(self, b) -> YoBvh:
        nodes = np.ascontiguousarray(b.nodes)
        pi = np.ascontiguousarray(b.primitive_indices, np.int32)
        prims = np.ascontiguousarray(b.primitives)
        self._keep += [nodes, pi, prims]
        return YoBvh(_p(nodes), nodes.size, _p(pi), pi.size, _p(prims), prims.size)

    def trace(self, rays: np.ndarray, threads: int = 0, stats: bool = True):
        """Closest hit for (N, 8) rays -> (YO_HIT_DTYPE array, stats (3, N))."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        hits = np.empty(n, YO_HIT_DTYPE)
        st = np.zeros((3, n), np.uint32) if stats else None
        threads = threads or (os.cpu_count() or 1)
        L = oracle_lib()
        sp = [None, None, None] if st is None else [st[0].ctypes.data, st[1].ctypes.data, st[2].ctypes.data]
        if self.two_level:
            L.yo_trace_two_level(C.byref(self.geo), C.byref(self.tl), rays.ctypes.data, n, hits.ctypes.data, *sp,
                                 threads)
        else:
            L.yo_trace_flat(C.byref(self.geo), C.byref(self.bvh), rays.ctypes.data, n, hits.ctypes.data, *sp,
                            threads)
        return hits, st

    def probe(self, rays: np.ndarray, targets: np.ndarray):
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        tg = np.ascontiguousarray(targets[:, :3], np.int32)
        counts = np.zeros(n, np.int32)
        ex = np.zeros(n, np.uint8)
        hits = np.zeros((n, 64), YO_HIT_DTYPE)
        oracle_lib().yo_probe(C.byref(self.geo), None if self.two_level else C.byref(self.bvh),
                              C.byref(self.tl) if self.two_level else None, rays.ctypes.data, n, tg.ctypes.data,
                              counts.ctypes.data, ex.ctypes.data, hits.ctypes.data)
        return hits, counts, ex


def oracle_sampler(kind: int, seed: int, spp: int, queries: np.ndarray, two_d: bool) -> np.ndarray:
    q = np.ascontiguousarray(queries, np.int32).reshape(-1, 6)
    out = np.empty(q.shape[0] * (2 if two_d else 1), np.float32)
    oracle_lib().yo_sampler(kind, seed, spp, q.ctypes.data, q.shape[0], int(two_d), out.ctypes.data)
    return out.reshape(-1, 2) if two_d else out


def oracle_rng(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, np.float32)
    oracle_lib().yo_rng_floats(seed, count, out.ctypes.data)
    return out


def oracle_seed_for_pixel_sample(seed: int, x: int, y: int, sample: int) -> int:
    return int(oracle_lib().yo_seed_for_pixel_sample(seed, x, y, sample))


def oracle_camera_rays(camera: np.ndarray, width: int, height: int, pixels: np.ndarray, samples: np.ndarray):
    cam = np.ascontiguousarray(camera, np.float32)
    px = np.ascontiguousarray(pixels, np.int32)
    sm = np.ascontiguousarray(samples, np.float32)
    out = np.empty((px.shape[0], 6), np.float32)
    oracle_lib().yo_camera_rays(cam.ctypes.data, width, height, px.ctypes.data, sm.ctypes.data, px.shape[0],
                                out.ctypes.data)
    return out


FILM_PIXEL_DTYPE = np.dtype([("sum", "<f4", 3), ("samples", "<u4"), ("luminance_mean", "<f4"),
                             ("luminance_m2", "<f4"), ("albedo_sum", "<f4", 3), ("normal_sum", "<f4", 3),
                             ("depth_sum", "<f4"), ("aov_samples", "<u4")])
assert FILM_PIXEL_DTYPE.itemsize == 56


def oracle_film(width: int, height: int, samples: np.ndarray):
    s = np.ascontiguousarray(samples, np.float32).reshape(-1, 13)
    px = np.zeros(width * height, FILM_PIXEL_DTYPE)
    bad = oracle_lib().yo_film_accumulate(width, height, s.ctypes.data, s.shape[0], px.ctypes.data)
    return px, int(bad)


# ----------------------------------------------------- compiled reference

_REF = None


def ref_lib() -> C.CDLL:
    global _REF
    if _REF is None:
        if not REF_SO.exists():
            raise FileNotFoundError(f"{REF_SO} not built (needs the reference sources; see oracle/Makefile)")
        L = C.CDLL(str(REF_SO))
        L.yrref_last_error.restype = C.c_char_p
        L.yrref_scene_create.restype = P
        L.yrref_scene_create.argtypes = [P, I64, P, I64, P, C.c_int, P, C.c_int, P, P, C.c_int]
        L.yrref_scene_destroy.argtypes = [P]
        L.yrref_scene_build.argtypes = [P, C.c_int, C.c_int, C.c_int]
        L.yrref_scene_is_two_level.argtypes = [P]
        L.yrref_flat_counts.argtypes = [P, P]
        L.yrref_flat_copy.argtypes = [P, P, P, P]
        L.yrref_two_level_counts.argtypes = [P, P]
        L.yrref_blas_counts.argtypes = [P, C.c_int, P]
        L.yrref_blas_copy.argtypes = [P, C.c_int, P, P, P, P, P]
        L.yrref_instances_copy.argtypes = [P, P, P, P, P, P]
        L.yrref_tlas_copy.argtypes = [P, P, P, P]
        L.yrref_trace.argtypes = [P, P, I64, P, P, P, P, P, P, P, P, P, P, P, C.c_int]
        L.yrref_trace_count.argtypes = [P, P, I64, C.c_int, P, P, C.c_int]
        L.yrref_trace_count.restype = I64
        L.yrref_probe.argtypes = [P, P, I64, P, P, P, P, P, P, P, P, P, P, C.c_int]
        L.yrref_sampler.argtypes = [C.c_int, U64, C.c_int, P, I64, C.c_int, P]
        L.yrref_seed_for_pixel_sample.argtypes = [U64, C.c_int, C.c_int, C.c_int]
        L.yrref_seed_for_pixel_sample.restype = U64
        L.yrref_rng_floats.argtypes = [U64, C.c_int, P]
        L.yrref_camera_rays.argtypes = [P, C.c_int, C.c_int, P, P, I64, P]
        L.yrref_film_accumulate.argtypes = [C.c_int, C.c_int, P, I64, P]
        L.yrref_film_accumulate.restype = U64
        L.yrref_texture_sample.argtypes = [C.c_int, C.c_int, P, C.c_int, C.c_int, C.c_int, P, P, I64, P]
        L.yrref_texture_mip_chain.argtypes = [C.c_int, C.c_int, P, C.c_int, C.c_int, P, P]
        L.yrref_texture_mip_chain.restype = C.c_int
        L.yrref_measured_eval.argtypes = [P, P, I64, P, P]
        L.yrref_measured_sample.argtypes = [P, P, I64, P]
        _REF = L
    return _REF


class RefScene:
    """The reference's own RenderSceneIR geometry + RenderAcceleration."""

    def __init__(self, geometry, split_method: str = "sah", max_leaf: int = 4, threads: int = 0):
        L = ref_lib()
        self._pos = np.ascontiguousarray(geometry.positions, np.float32)
        self._idx = np.ascontiguousarray(geometry.indices, np.uint32)
        prims = geometry.primitives
        self._prims = np.ascontiguousarray(
            np.stack([prims["first_index"], prims["index_count"]], 1) if prims.size else np.zeros((0, 2)), np.uint32)
        sp = geometry.spheres
        self._sph = np.ascontiguousarray(
            np.concatenate([sp["center"], sp["radius"][:, None]], 1) if sp.size else np.zeros((0, 4)), np.float32)
        inst = geometry.instances
        self._ip = np.ascontiguousarray(inst["primitive"], np.int32)
        self._im = np.ascontiguousarray(inst["object_to_world"].reshape(-1, 16), np.float32)
        self.h = L.yrref_scene_create(_p(self._pos), self._pos.shape[0], _p(self._idx), self._idx.size,
                                      _p(self._prims), self._prims.shape[0], _p(self._sph), self._sph.shape[0],
                                      _p(self._ip), _p(self._im), self._ip.size)
        self.errors = L.yrref_scene_build(self.h, 1 if split_method == "median" else 0, max_leaf, threads)
        self.error = L.yrref_last_error().decode() if self.errors else ""
        self.two_level = bool(L.yrref_scene_is_two_level(self.h))

    def __del__(self):
        try:
            ref_lib().yrref_scene_destroy(self.h)
        except Exception:
            pass

    @staticmethod
    def _bvh_arrays(counts):
        from yaoray_b200._lib import BVH_PRIM_DTYPE, NODE_DTYPE
        return (np.zeros(counts[0], NODE_DTYPE), np.zeros(counts[1], np.int32), np.zeros(counts[2], BVH_PRIM_DTYPE))

    def flat_bvh(self):
        """(nodes, primitive_indices, primitives, max_depth) of the flat BVH."""
        L = ref_lib()
        c = np.zeros(4, np.int64)
        L.yrref_flat_counts(self.h, c.ctypes.data)
        nodes, pi, prims = self._bvh_arrays(c)
        L.yrref_flat_copy(self.h, _p(nodes), _p(pi), _p(prims))
        return nodes, pi, prims, int(c[3])

    def two_level_bvh(self):
        """dict with blases, instances and tlas arrays of the TwoLevelBvh."""
        from yaoray_b200._lib import NODE_DTYPE
        L = ref_lib()
        c = np.zeros(6, np.int64)
        L.yrref_two_level_counts(self.h, c.ctypes.data)
        blases = []
        for b in range(int(c[0])):
            bc = np.zeros(4, np.int64)
            L.yrref_blas_counts(self.h, b, bc.ctypes.data)
            nodes, pi, prims = self._bvh_arrays(bc)
            bounds = np.zeros(6, np.float32)
            mp = np.zeros(1, np.int32)
            L.yrref_blas_copy(self.h, b, _p(nodes), _p(pi), _p(prims), bounds.ctypes.data, mp.ctypes.data)
            blases.append((int(mp[0]), bounds.reshape(2, 3), nodes, pi, prims, int(bc[3])))
        n = int(c[1])
        ip = np.zeros(n, np.int32)
        ib = np.zeros(n, np.int32)
        o2w = np.zeros((n, 16), np.float32)
        w2o = np.zeros((n, 16), np.float32)
        wb = np.zeros((n, 6), np.float32)
        if n:
            L.yrref_instances_copy(self.h, ip.ctypes.data, ib.ctypes.data, o2w.ctypes.data, w2o.ctypes.data,
                                   wb.ctypes.data)
        tn = np.zeros(int(c[2]), NODE_DTYPE)
        tpi = np.zeros(int(c[3]), np.int32)
        tpr = np.zeros((int(c[4]), 3), np.int32)
        L.yrref_tlas_copy(self.h, _p(tn), _p(tpi), _p(tpr))
        return {"blases": blases, "instance_primitive": ip, "instance_blas": ib, "object_to_world": o2w,
                "world_to_object": w2o, "world_bounds": wb, "tlas_nodes": tn, "tlas_primitive_indices": tpi,
                "tlas_primitives": tpr, "tlas_max_depth": int(c[5])}

    def trace(self, rays: np.ndarray, threads: int = 0):
        """IntersectAcceleration over (N, 8) rays -> dict of per-ray arrays."""
        L = ref_lib()
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        out = {k: np.empty(n, dt) for k, dt in [("t", np.float32), ("triangle_index", np.int32),
                                                ("sphere", np.int32), ("mesh_primitive", np.int32),
                                                ("instance", np.int32), ("u", np.float32), ("v", np.float32),
                                                ("hit", np.uint8), ("node_tests", np.uint32),
                                                ("triangle_tests", np.uint32), ("sphere_tests", np.uint32)]}
        L.yrref_trace(self.h, rays.ctypes.data, n, *[out[k].ctypes.data for k in
                      ["t", "triangle_index", "sphere", "mesh_primitive", "instance", "u", "v", "hit",
                       "node_tests", "triangle_tests", "sphere_tests"]], threads)
        return out

    def trace_count(self, rays: np.ndarray, any_hit: bool, threads: int = 0, t_out=None, id_out=None) -> int:
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        return int(ref_lib().yrref_trace_count(self.h, rays.ctypes.data, rays.shape[0], int(any_hit),
                                               _p(t_out), _p(id_out), threads))

    def probe(self, rays: np.ndarray, targets: np.ndarray, threads: int = 1):
        L = ref_lib()
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = rays.shape[0]
        tp = np.ascontiguousarray(targets[:, 0], np.int32)
        ti = np.ascontiguousarray(targets[:, 1], np.int32)
        ts = np.ascontiguousarray(targets[:, 2], np.int32)
        counts = np.zeros(n, np.int32)
        ex = np.zeros(n, np.uint8)
        t = np.zeros((n, 64), np.float32)
        tri = np.full((n, 64), -1, np.int32)
        inst = np.full((n, 64), -1, np.int32)
        u = np.zeros((n, 64), np.float32)
        v = np.zeros((n, 64), np.float32)
        L.yrref_probe(self.h, rays.ctypes.data, n, tp.ctypes.data, ti.ctypes.data, ts.ctypes.data, counts.ctypes.data,
                      ex.ctypes.data, t.ctypes.data, tri.ctypes.data, inst.ctypes.data, u.ctypes.data, v.ctypes.data,
                      threads)
        return {"count": counts, "exhausted": ex, "t": t, "triangle_index": tri, "instance": inst, "u": u, "v": v}


def ref_sampler(kind: int, seed: int, spp: int, queries: np.ndarray, two_d: bool) -> np.ndarray:
    q = np.ascontiguousarray(queries, np.int32).reshape(-1, 6)
    out = np.empty(q.shape[0] * (2 if two_d else 1), np.float32)
    ref_lib().yrref_sampler(kind, seed, spp, q.ctypes.data, q.shape[0], int(two_d), out.ctypes.data)
    return out.reshape(-1, 2) if two_d else out


def _texture_args(texels, uvs, footprints):
    tx = np.ascontiguousarray(texels, np.float32)
    uv = np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
    fp = None if footprints is None else np.ascontiguousarray(footprints, np.float32).reshape(-1, 4)
    return tx, uv, fp


def _mip_buffers(width: int, height: int):
    return np.zeros((max(width * height, 0) + 64) * 4, np.float32), np.zeros(80, np.int32)


def _mip_levels(out, dims, count):
    levels, at = [], 0
    for k in range(count):
        w, h = int(dims[2 * k]), int(dims[2 * k + 1])
        levels.append(out[4 * at:4 * (at + w * h)].reshape(h, w, 4).copy())
        at += w * h
    return levels


def ref_texture_sample(texels: np.ndarray, filter: int, wrap_s: int, wrap_t: int, uvs: np.ndarray,
                       footprints: np.ndarray | None = None) -> np.ndarray:
    """The reference's SampleTexture4 on an (h, w, 4) RGBA32F image."""
    tx, uv, fp = _texture_args(texels, uvs, footprints)
    out = np.empty((uv.shape[0], 4), np.float32)
    h, w = (tx.shape[0], tx.shape[1]) if tx.ndim == 3 else (0, 0)
    ref_lib().yrref_texture_sample(w, h, tx.ctypes.data if tx.size else None, filter, wrap_s, wrap_t,
                                   uv.ctypes.data, None if fp is None else fp.ctypes.data, uv.shape[0],
                                   out.ctypes.data)
    return out


def ref_texture_mip_chain(texels: np.ndarray, wrap_s: int, wrap_t: int) -> list:
    """The reference's BuildTextureMipChain levels (after the image)."""
    tx = np.ascontiguousarray(texels, np.float32)
    h, w = tx.shape[0], tx.shape[1]
    out, dims = _mip_buffers(w, h)
    count = ref_lib().yrref_texture_mip_chain(w, h, tx.ctypes.data, wrap_s, wrap_t, out.ctypes.data,
                                              dims.ctypes.data)
    return _mip_levels(out, dims, count)


def oracle_texture_sample(texels: np.ndarray, filter: int, wrap_s: int, wrap_t: int, uvs: np.ndarray,
                          footprints: np.ndarray | None = None) -> np.ndarray:
    """The C restatement's SampleTexture4 on an (h, w, 4) RGBA32F image."""
    tx, uv, fp = _texture_args(texels, uvs, footprints)
    out = np.empty((uv.shape[0], 4), np.float32)
    h, w = (tx.shape[0], tx.shape[1]) if tx.ndim == 3 else (0, 0)
    oracle_lib().yo_texture_sample(w, h, tx.ctypes.data if tx.size else None, filter, wrap_s, wrap_t,
                                   uv.ctypes.data, None if fp is None else fp.ctypes.data, uv.shape[0],
                                   out.ctypes.data)
    return out


def oracle_texture_mip_chain(texels: np.ndarray, wrap_s: int, wrap_t: int) -> list:
    """The C restatement's BuildTextureMipChain levels (after the image)."""
    tx = np.ascontiguousarray(texels, np.float32)
    h, w = tx.shape[0], tx.shape[1]
    out, dims = _mip_buffers(w, h)
    count = oracle_lib().yo_texture_mip_chain(w, h, tx.ctypes.data, wrap_s, wrap_t, out.ctypes.data,
                                              dims.ctypes.data)
    return _mip_levels(out, dims, count)


def ref_measured_eval(brdf, wo, wi, n):
    """The reference's EvaluateMeasured / PdfMeasured (brdf: a
    yaoray_b200.measured.MeasuredBrdf): (f (n, 3), pdf (n,))."""
    q = np.ascontiguousarray(np.concatenate([np.reshape(wo, (-1, 3)), np.reshape(wi, (-1, 3)),
                                             np.reshape(n, (-1, 3))], 1), np.float32)
    f = np.empty((q.shape[0], 3), np.float32)
    pdf = np.empty(q.shape[0], np.float32)
    st, keep = brdf.c_struct()
    ref_lib().yrref_measured_eval(C.addressof(st), q.ctypes.data, q.shape[0], f.ctypes.data, pdf.ctypes.data)
    del keep
    return f, pdf


def ref_measured_sample(brdf, wo, n, u):
    """The reference's SampleMeasured: (n, 8) rows of wi, weight, pdf, valid."""
    q = np.ascontiguousarray(np.concatenate([np.reshape(wo, (-1, 3)), np.reshape(n, (-1, 3)),
                                             np.reshape(u, (-1, 2))], 1), np.float32)
    out = np.empty((q.shape[0], 8), np.float32)
    st, keep = brdf.c_struct()
    ref_lib().yrref_measured_sample(C.addressof(st), q.ctypes.data, q.shape[0], out.ctypes.data)
    del keep
    return out


def ref_bssrdf_table(g: float, eta: float, rho_count: int = 100, radius_count: int = 64) -> dict:
    """The reference's ComputeBeamDiffusionBSSRDF table."""
    L = ref_lib()
    t = {"rho_samples": np.zeros(rho_count, np.float32), "radius_samples": np.zeros(radius_count, np.float32),
         "profile": np.zeros(rho_count * radius_count, np.float32), "rho_eff": np.zeros(rho_count, np.float32),
         "profile_cdf": np.zeros(rho_count * radius_count, np.float32)}
    L.yrref_bssrdf_table.argtypes = [C.c_float, C.c_float, C.c_int, C.c_int, P, P, P, P, P]
    L.yrref_bssrdf_table(g, eta, rho_count, radius_count, _p(t["rho_samples"]), _p(t["radius_samples"]),
                         _p(t["profile"]), _p(t["rho_eff"]), _p(t["profile_cdf"]))
    return t


def ref_bsdf_eval(material, wo, wi, n, seeds):
    """The reference's EvaluateBsdf then PdfBsdf (one RenderMaterial from a
    MATERIAL_DTYPE record) with Rng(seeds[i]) per row: (f (n, 3), pdf (n,))."""
    from yaoray_b200.render import MATERIAL_DTYPE
    m = np.ascontiguousarray(np.asarray(material, MATERIAL_DTYPE).reshape(1))
    q = np.ascontiguousarray(np.concatenate([np.reshape(wo, (-1, 3)), np.reshape(wi, (-1, 3)),
                                             np.reshape(n, (-1, 3))], 1), np.float32)
    s = np.ascontiguousarray(seeds, np.uint64).reshape(-1)
    f = np.empty((q.shape[0], 3), np.float32)
    pdf = np.empty(q.shape[0], np.float32)
    L = ref_lib()
    L.yrref_bsdf_eval.argtypes = [P, P, P, I64, P, P]
    L.yrref_bsdf_eval(m.ctypes.data, q.ctypes.data, s.ctypes.data, q.shape[0], f.ctypes.data, pdf.ctypes.data)
    return f, pdf


def ref_bsdf_sample(material, wo, n, u, seeds) -> np.ndarray:
    """The reference's SampleBsdf with Rng(seeds[i]) per row: (n, 9) rows of
    wi, weight, pdf, valid, specular."""
    from yaoray_b200.render import MATERIAL_DTYPE
    m = np.ascontiguousarray(np.asarray(material, MATERIAL_DTYPE).reshape(1))
    q = np.ascontiguousarray(np.concatenate([np.reshape(wo, (-1, 3)), np.reshape(n, (-1, 3)),
                                             np.reshape(u, (-1, 2))], 1), np.float32)
    s = np.ascontiguousarray(seeds, np.uint64).reshape(-1)
    out = np.empty((q.shape[0], 9), np.float32)
    L = ref_lib()
    L.yrref_bsdf_sample.argtypes = [P, P, P, I64, P]
    L.yrref_bsdf_sample(m.ctypes.data, q.ctypes.data, s.ctypes.data, q.shape[0], out.ctypes.data)
    return out


def ref_bssrdf_eval(sigma_a, sigma_s, eta: float, channels, u, r, g: float = 0.0):
    """The reference TabulatedBSSRDF (100 x 64 table for g, eta):
    (Sample_Sr(ch, u), Pdf_Sr(ch, r), Sr(r) (n, 3)) per row."""
    ch = np.ascontiguousarray(channels, np.int32).reshape(-1)
    uu = np.ascontiguousarray(u, np.float32).reshape(-1)
    rr = np.ascontiguousarray(r, np.float32).reshape(-1)
    n = ch.size
    sa = np.ascontiguousarray(sigma_a, np.float32)
    ss = np.ascontiguousarray(sigma_s, np.float32)
    sample_r, pdf, sr = np.empty(n, np.float32), np.empty(n, np.float32), np.empty((n, 3), np.float32)
    L = ref_lib()
    L.yrref_bssrdf_eval.argtypes = [P, P, C.c_float, C.c_float, C.c_int, P, P, P, P, P, P]
    L.yrref_bssrdf_eval(sa.ctypes.data, ss.ctypes.data, eta, g, n, ch.ctypes.data, uu.ctypes.data, rr.ctypes.data,
                        sample_r.ctypes.data, pdf.ctypes.data, sr.ctypes.data)
    return sample_r, pdf, sr


def ref_bssrdf_pdf_sp(sigma_a, sigma_s, eta: float, queries, g: float = 0.0) -> np.ndarray:
    """The reference TabulatedBSSRDF::Pdf_Sp per row of (po, ss, ts, ns, pi, ni)."""
    q = np.ascontiguousarray(queries, np.float32).reshape(-1, 18)
    sa = np.ascontiguousarray(sigma_a, np.float32)
    ss = np.ascontiguousarray(sigma_s, np.float32)
    out = np.empty(q.shape[0], np.float32)
    L = ref_lib()
    L.yrref_bssrdf_pdf_sp.argtypes = [P, P, C.c_float, C.c_float, C.c_int, P, P]
    L.yrref_bssrdf_pdf_sp(sa.ctypes.data, ss.ctypes.data, eta, g, q.shape[0], q.ctypes.data, out.ctypes.data)
    return out


def ref_rng(seed: int, count: int) -> np.ndarray:
    out = np.empty(count, np.float32)
    ref_lib().yrref_rng_floats(seed, count, out.ctypes.data)
    return out


def ref_seed_for_pixel_sample(seed: int, x: int, y: int, sample: int) -> int:
    return int(ref_lib().yrref_seed_for_pixel_sample(seed, x, y, sample))


def ref_camera_rays(camera, width, height, pixels, samples):
    cam = np.ascontiguousarray(camera, np.float32)
    px = np.ascontiguousarray(pixels, np.int32)
    sm = np.ascontiguousarray(samples, np.float32)
    out = np.empty((px.shape[0], 6), np.float32)
    ref_lib().yrref_camera_rays(cam.ctypes.data, width, height, px.ctypes.data, sm.ctypes.data, px.shape[0],
                                out.ctypes.data)
    return out


def ref_film(width: int, height: int, samples: np.ndarray):
    s = np.ascontiguousarray(samples, np.float32).reshape(-1, 13)
    px = np.zeros(width * height, FILM_PIXEL_DTYPE)
    bad = ref_lib().yrref_film_accumulate(width, height, s.ctypes.data, s.shape[0], px.ctypes.data)
    return px, int(bad)


# ------------------------------------------------ reference renders (CPU)

def _bind_jobs(L):
    if getattr(L, "_jobs_bound", False):
        return L
    L.yrref_pbrt_load.restype = P
    L.yrref_pbrt_load.argtypes = [C.c_char_p]
    L.yrref_job_destroy.argtypes = [P]
    L.yrref_job_counts.argtypes = [P, P]
    L.yrref_job_geometry.argtypes = [P, P, P, P, P, P]
    L.yrref_job_materials.argtypes = [P, P]
    L.yrref_job_lights.argtypes = [P, P, P, P, P, P, P]
    L.yrref_job_from_desc.restype = P
    L.yrref_job_from_desc.argtypes = [P]
    L.yrref_job_render.argtypes = [P, C.c_int, C.c_int, P, P, P]
    L.yrref_job_render_resume.argtypes = [P, C.c_int, C.c_int, P, C.c_int, P, P, P]
    L._jobs_bound = True
    return L


class RefJob:
    """A RenderJob of the reference: loaded from a PBRT file by its own
    frontend, or assembled from a RenderScene; rendered by its CpuBackend."""

    def __init__(self, handle):
        self.h = handle

    @staticmethod
    def load_pbrt(path) -> "RefJob":
        L = _bind_jobs(ref_lib())
        h = L.yrref_pbrt_load(str(path).encode())
        if not h:
            raise RuntimeError(L.yrref_last_error().decode())
        return RefJob(h)

    @staticmethod
    def from_scene(scene) -> "RefJob":
        from yaoray_b200.render import scene_desc
        L = _bind_jobs(ref_lib())
        desc, keep = scene_desc(scene)
        h = L.yrref_job_from_desc(C.addressof(desc))
        del keep
        return RefJob(h)

    def __del__(self):
        try:
            _bind_jobs(ref_lib()).yrref_job_destroy(self.h)
        except Exception:
            pass

    def export(self):
        """The compiled RenderSceneIR + settings as a yaoray_b200 RenderScene."""
        from yaoray_b200 import _lib
        from yaoray_b200.accel import SceneGeometry
        from yaoray_b200.render import EMISSIVE_DTYPE, MATERIAL_DTYPE, Camera, RenderScene, Settings
        L = _bind_jobs(ref_lib())
        c = np.zeros(11, np.int64)
        L.yrref_job_counts(self.h, c.ctypes.data)
        nv, ni, npr, ns, nin, nm, ne = (int(x) for x in c[:7])
        verts = np.zeros((nv, 12), np.float32)
        idx = np.zeros(ni, np.uint32)
        prims = np.zeros(npr, _lib.PRIM_DTYPE)
        sph = np.zeros(ns, _lib.SPHERE_DTYPE)
        inst = np.zeros(nin, _lib.INSTANCE_DTYPE)
        L.yrref_job_geometry(self.h, _p(verts), _p(idx), _p(prims), _p(sph), _p(inst))
        mats = np.zeros(nm, MATERIAL_DTYPE)
        L.yrref_job_materials(self.h, _p(mats))
        em = np.zeros(ne, EMISSIVE_DTYPE)
        na = int(c[10])
        prob = np.zeros(na, np.float32)
        alias = np.zeros(na, np.int32)
        pmf = np.zeros(na, np.float32)
        cam = Camera()
        st = Settings()
        L.yrref_job_lights(self.h, _p(em), _p(prob), _p(alias), _p(pmf), C.addressof(cam), C.addressof(st))
        geom = SceneGeometry(verts[:, 0:3], idx, prims, sph, inst)
        camd = {"origin": tuple(cam.origin), "forward": tuple(cam.forward), "right": tuple(cam.right),
                "up": tuple(cam.up), "fov_y_radians": cam.fov_y_radians}
        return RenderScene(geom, mats, camd, st.width, st.height, spp=st.spp, max_depth=st.max_depth, seed=st.seed,
                           sampler=st.sampler, radiance_clamp=st.radiance_clamp,
                           normals=verts[:, 3:6].copy() if (prims["flags"] & 1).any() else None, emissive=em,
                           uvs=verts[:, 6:8].copy() if (prims["flags"] & 2).any() else None,
                           tangents=verts[:, 8:12].copy() if (prims["flags"] & 4).any() else None,
                           alias=(prob, alias, pmf) if na else None,
                           adaptive={"enabled": bool(st.adaptive_enabled), "min_spp": st.adaptive_min_spp,
                                     "relative_error": st.adaptive_relative_error,
                                     "absolute_error": st.adaptive_absolute_error,
                                     "confidence": st.adaptive_confidence})

    def shadow_visibility(self, rays: np.ndarray) -> np.ndarray:
        """The reference's TraceShadowVisibility on this job's scene (prepared
        as the CPU backend prepares it) for (n, 8) rays (origin, unused,
        direction, max_distance) -> (n, 4): RGB transmittance, visible."""
        L = _bind_jobs(ref_lib())
        L.yrref_job_shadow_visibility.argtypes = [P, P, I64, P]
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 4), np.float32)
        if L.yrref_job_shadow_visibility(self.h, r.ctypes.data, r.shape[0], out.ctypes.data) != 0:
            raise RuntimeError(L.yrref_last_error().decode())
        return out

    def render(self, threads: int = 0, spp: int = 0, resume_film=None, resume_spp: int = 0):
        """CpuBackend render -> (film FILM_PIXEL_DTYPE (H*W), stats dict, seconds).
        With `resume_film` (FILM_PIXEL_DTYPE, H x W) the render resumes from it
        after `resume_spp` passes, and the stats carry converged_pixels."""
        L = _bind_jobs(ref_lib())
        c = np.zeros(11, np.int64)
        L.yrref_job_counts(self.h, c.ctypes.data)
        from yaoray_b200.render import Settings
        cam_dummy = None  # noqa: F841
        st = Settings()
        from yaoray_b200.render import Camera
        cam = Camera()
        em = np.zeros(max(int(c[6]), 1), np.dtype([("a", "<i4"), ("b", "<f4", 4)]))
        na = max(int(c[10]), 1)
        L.yrref_job_lights(self.h, _p(em), _p(np.zeros(na, np.float32)), _p(np.zeros(na, np.int32)),
                           _p(np.zeros(na, np.float32)), C.addressof(cam), C.addressof(st))
        film = np.zeros(st.width * st.height, FILM_PIXEL_DTYPE)
        stats = np.zeros(8, np.uint64)
        secs = C.c_double()
        keys = ["samples_rendered", "rays_traced", "shadow_rays", "occluded_shadow_rays", "hits", "misses",
                "bad_samples"]
        if resume_film is None:
            rc = L.yrref_job_render(self.h, threads, spp, film.ctypes.data, stats.ctypes.data, C.byref(secs))
        else:
            resume = np.ascontiguousarray(resume_film, FILM_PIXEL_DTYPE).reshape(-1)
            assert resume.size == film.size
            rc = L.yrref_job_render_resume(self.h, threads, spp, resume.ctypes.data, resume_spp, film.ctypes.data,
                                           stats.ctypes.data, C.byref(secs))
            keys.append("converged_pixels")
        if rc != 0:
            raise RuntimeError(L.yrref_last_error().decode())
        return film.reshape(st.height, st.width), dict(zip(keys, map(int, stats))), float(secs.value)
