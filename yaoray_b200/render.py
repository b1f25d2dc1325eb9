"""Render path — the Python mirror of the reference's backend interface
(include/yaoray/runtime/backend.hpp:90-98) over libyrcuda's render ABI.

    backend = CudaBackend()                       # RenderBackend for RenderBackendKind::Cuda
    prepared = backend.prepare(scene)             # RenderBackend::Prepare(RenderJob)
    result = backend.render(prepared, request)    # RenderBackend::Render(PreparedScene, RenderRequest)

`RenderScene` holds a RenderSceneIR + RenderSettings as numpy arrays (the
reference IR's fields, textures, measured BRDFs and analytic lights
included). Errors come
back as `RenderResult(ok=False, error=...)` like the reference's result
structs; programming errors raise `YrcError`.
"""
from __future__ import annotations

import dataclasses

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import YrcError, check, lib, ptr
from .accel import SceneGeometry, build_bvh, build_bvh_device, build_two_level_bvh
from .measured import measured_array
from .texture import textures_array

# --------------------------------------------------------------- C mirrors


class Material(C.Structure):
    _fields_ = [("kind", C.c_int32), ("reflectance", C.c_float * 3), ("eta", C.c_float * 3), ("k", C.c_float * 3),
                ("ior", C.c_float), ("uroughness", C.c_float), ("vroughness", C.c_float),
                ("remap_roughness", C.c_int32), ("mix_material_a", C.c_int32), ("mix_material_b", C.c_int32),
                ("mix_amount", C.c_float), ("coating_ior", C.c_float), ("coating_roughness", C.c_float),
                ("coat_thickness", C.c_float), ("coat_absorption", C.c_float * 3), ("coat_maxdepth", C.c_int32),
                ("coat_nsamples", C.c_int32), ("sigma_a", C.c_float * 3), ("sigma_s", C.c_float * 3),
                ("bssrdf_eta", C.c_float), ("bssrdf_index", C.c_int32), ("emission", C.c_float * 3),
                ("alpha", C.c_float), ("absorption_color", C.c_float * 3), ("absorption_distance", C.c_float),
                ("reflectance_texture", C.c_int32), ("alpha_texture", C.c_int32), ("normal_map", C.c_int32),
                ("measured_index", C.c_int32), ("normal_scale", C.c_float)]


MATERIAL_DTYPE = np.dtype([("kind", "<i4"), ("reflectance", "<f4", 3), ("eta", "<f4", 3), ("k", "<f4", 3),
                           ("ior", "<f4"), ("uroughness", "<f4"), ("vroughness", "<f4"), ("remap_roughness", "<i4"),
                           ("mix_material_a", "<i4"), ("mix_material_b", "<i4"), ("mix_amount", "<f4"),
                           ("coating_ior", "<f4"), ("coating_roughness", "<f4"), ("coat_thickness", "<f4"),
                           ("coat_absorption", "<f4", 3), ("coat_maxdepth", "<i4"), ("coat_nsamples", "<i4"),
                           ("sigma_a", "<f4", 3), ("sigma_s", "<f4", 3), ("bssrdf_eta", "<f4"),
                           ("bssrdf_index", "<i4"), ("emission", "<f4", 3), ("alpha", "<f4"),
                           ("absorption_color", "<f4", 3), ("absorption_distance", "<f4"),
                           ("reflectance_texture", "<i4"), ("alpha_texture", "<i4"), ("normal_map", "<i4"),
                           ("measured_index", "<i4"), ("normal_scale", "<f4")])
assert MATERIAL_DTYPE.itemsize == C.sizeof(Material)

EMISSIVE_DTYPE = np.dtype([("primitive_index", "<i4"), ("radiance", "<f4", 3), ("area", "<f4")])
# AnalyticLight (include/yaoray/scene/light.hpp:38-45); kind 0 point, 1 spot, 2 distant.
ANALYTIC_DTYPE = np.dtype([("kind", "<i4"), ("position", "<f4", 3), ("direction", "<f4", 3), ("intensity", "<f4", 3),
                           ("cone_angle", "<f4"), ("cone_cos_inner", "<f4")])
FILM_PIXEL_DTYPE = np.dtype([("sum", "<f4", 3), ("samples", "<u4"), ("luminance_mean", "<f4"),
                             ("luminance_m2", "<f4"), ("albedo_sum", "<f4", 3), ("normal_sum", "<f4", 3),
                             ("depth_sum", "<f4"), ("aov_samples", "<u4")])
assert FILM_PIXEL_DTYPE.itemsize == 56

# RenderMaterialKind
DIFFUSE, CONDUCTOR, DIELECTRIC, THIN_DIELECTRIC, COATED_DIFFUSE, COATED_CONDUCTOR = 0, 1, 2, 3, 4, 5
DIFFUSE_TRANSMISSION, MIX, MEASURED, SUBSURFACE, SUBSURFACE_EXIT = 6, 7, 8, 9, 10
# RenderSamplerKind
INDEPENDENT, STRATIFIED, OWEN_SOBOL, ZSOBOL = 0, 1, 2, 3


def default_material(**kw) -> np.void:
    """A RenderMaterial with the reference's defaults (material.hpp:31-65)."""
    m = np.zeros(1, MATERIAL_DTYPE)[0]
    m["kind"] = DIFFUSE
    m["reflectance"] = (0.5, 0.5, 0.5)
    m["ior"] = 1.5
    m["remap_roughness"] = 1
    m["mix_material_a"] = m["mix_material_b"] = -1
    m["mix_amount"] = 0.5
    m["coating_ior"] = 1.5
    m["coat_thickness"] = 0.01
    m["coat_maxdepth"] = 10
    m["coat_nsamples"] = 1
    m["bssrdf_eta"] = 1.33
    m["bssrdf_index"] = -1
    m["alpha"] = 1.0
    m["absorption_color"] = (1.0, 1.0, 1.0)
    m["absorption_distance"] = 1.0
    m["reflectance_texture"] = m["alpha_texture"] = m["normal_map"] = m["measured_index"] = -1
    m["normal_scale"] = 1.0
    for k, v in kw.items():
        m[k] = v
    return m


class AliasTable(C.Structure):
    _fields_ = [("probability", C.c_void_p), ("alias", C.c_void_p), ("pmf", C.c_void_p), ("count", C.c_int32)]


class AnalyticLight(C.Structure):
    _fields_ = [("kind", C.c_int32), ("position", C.c_float * 3), ("direction", C.c_float * 3),
                ("intensity", C.c_float * 3), ("cone_angle", C.c_float), ("cone_cos_inner", C.c_float)]


class Environment(C.Structure):
    _fields_ = [("active", C.c_int32), ("radiance", C.c_float * 3), ("strength", C.c_float),
                ("rotation_radians", C.c_float), ("width", C.c_int32), ("height", C.c_int32),
                ("texels", C.c_void_p), ("texel_weights", C.c_void_p), ("row_weights", C.c_void_p),
                ("row_cdf", C.c_void_p), ("conditional_cdfs", C.c_void_p), ("total_weight", C.c_float)]


class BssrdfTable(C.Structure):
    _fields_ = [("rho_count", C.c_int32), ("radius_count", C.c_int32), ("rho_samples", C.c_void_p),
                ("radius_samples", C.c_void_p), ("profile", C.c_void_p), ("rho_eff", C.c_void_p),
                ("profile_cdf", C.c_void_p)]


class Camera(C.Structure):
    _fields_ = [("origin", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("fov_y_radians", C.c_float)]


class Settings(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("spp", C.c_int32), ("max_depth", C.c_int32),
                ("seed", C.c_uint64), ("sampler", C.c_int32), ("radiance_clamp", C.c_float),
                ("adaptive_enabled", C.c_int32), ("adaptive_min_spp", C.c_int32),
                ("adaptive_relative_error", C.c_float), ("adaptive_absolute_error", C.c_float),
                ("adaptive_confidence", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [("geometry", _lib.Geometry), ("normals", C.c_void_p), ("normal_stride", C.c_int64),
                ("materials", C.c_void_p), ("material_count", C.c_int32), ("emissive", C.c_void_p),
                ("emissive_count", C.c_int32), ("emissive_power", AliasTable), ("analytic", C.c_void_p),
                ("analytic_count", C.c_int32), ("analytic_power", AliasTable), ("environment", Environment),
                ("bssrdf_tables", C.c_void_p), ("bssrdf_count", C.c_int32), ("camera", Camera),
                ("settings", Settings), ("flat", C.c_void_p), ("two_level", C.c_void_p),
                ("uvs", C.c_void_p), ("uv_stride", C.c_int64), ("tangents", C.c_void_p),
                ("tangent_stride", C.c_int64), ("textures", C.c_void_p), ("texture_count", C.c_int32),
                ("measured", C.c_void_p), ("measured_count", C.c_int32)]


class Progress(C.Structure):
    _fields_ = [("completed_spp", C.c_int32), ("target_spp", C.c_int32), ("completed_samples", C.c_uint64),
                ("target_samples", C.c_uint64), ("active_pixels", C.c_uint64), ("converged_pixels", C.c_uint64),
                ("rays_traced", C.c_uint64), ("elapsed_seconds", C.c_double)]


PROGRESS_FN = C.CFUNCTYPE(C.c_int32, C.POINTER(Progress), C.c_void_p, C.c_uint64, C.c_void_p, C.c_void_p,
                          C.c_size_t)


class Request(C.Structure):
    _fields_ = [("resume_film", C.c_void_p), ("resume_bad_samples", C.c_uint64),
                ("resume_completed_spp", C.c_int32), ("stop_flag", C.c_void_p), ("progress", PROGRESS_FN),
                ("user", C.c_void_p)]


class Stats(C.Structure):
    _fields_ = [("samples_rendered", C.c_uint64), ("converged_pixels", C.c_uint64), ("rays_traced", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("occluded_shadow_rays", C.c_uint64), ("triangle_tests", C.c_uint64),
                ("sphere_tests", C.c_uint64), ("bvh_node_tests", C.c_uint64), ("bvh_nodes", C.c_int32),
                ("bvh_max_depth", C.c_int32), ("hits", C.c_uint64), ("misses", C.c_uint64),
                ("bad_samples", C.c_uint64), ("threads", C.c_int32), ("elapsed_seconds", C.c_double),
                ("device_seconds", C.c_double), ("cache_queries", C.c_uint64), ("cache_records", C.c_uint64),
                ("kernel_launches", C.c_uint64)]


class RenderTuning(C.Structure):
    """yrc_render_tuning: the configuration the render autotuner chose."""
    _fields_ = [("capacity", C.c_int64), ("trace_shape", C.c_int32), ("candidates", C.c_int32),
                ("seconds_per_sample", C.c_double)]


TUNE_CAPACITY = 1
TUNE_TRACE_SHAPE = 2


class CacheSettings(C.Structure):
    """yrc_cache_settings: how the path tracer uses an attached radiance cache."""
    _fields_ = [("spread_threshold", C.c_float), ("train_one_in", C.c_int32), ("train_records", C.c_int32),
                ("train", C.c_int32), ("train_steps", C.c_int32), ("delta_vertices", C.c_int32),
                ("averaged", C.c_int32)]


def _bind():
    L = lib()
    if getattr(L, "_render_bound", False):
        return L
    P = C.c_void_p
    for name, res, args in [
        ("yrc_render_scene_create", C.c_int, [P, P]),
        ("yrc_render_scene_destroy", None, [P]),
        ("yrc_render_scene_device_bytes", C.c_int64, [P]),
        ("yrc_render", C.c_int, [P, P, P, P, P]),
        ("yrc_render_scene_set_cache", C.c_int, [P, P, P]),
        ("yrc_render_scene_set_capacity", C.c_int, [P, C.c_int64]),
        ("yrc_render_scene_capacity", C.c_int64, [P]),
        ("yrc_render_autotune", C.c_int, [P, C.c_int32, P]),
        ("yrc_render_scene_set_tuning", C.c_int, [P, P]),
        ("yrc_render_scene_shadow_eval", C.c_int, [P, P, C.c_int64, P]),
        ("yrc_render_scene_set_view", C.c_int, [P, P, C.c_uint64]),
        ("yrc_render_many", C.c_int, [P, C.c_int32, P, P, P, P, P]),
        ("yrc_render_pooled", C.c_int, [P, C.c_int32, P, P, P, P, P]),
        ("yrc_bssrdf_table_build", C.c_int, [C.c_float, C.c_float, C.c_int32, C.c_int32, P, P, P, P, P]),
        ("yrc_alias_table_build", C.c_int, [P, C.c_int32, P, P, P]),
        ("yrc_environment_distribution_build", C.c_int, [P, C.c_int32, C.c_int32, P, P, P, P, P]),
    ]:
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L._render_bound = True
    return L


# ------------------------------------------------------------------ scene


@dataclass
class EnvironmentMap:
    """RenderEnvironment + its RGBA32F texture and distribution."""

    active: bool = False
    radiance: tuple = (0.0, 0.0, 0.0)
    strength: float = 1.0
    rotation: float = 0.0
    texels: np.ndarray | None = None   # (H, W, 4) float32
    texel_weights: np.ndarray | None = None
    row_weights: np.ndarray | None = None
    row_cdf: np.ndarray | None = None
    conditional_cdfs: np.ndarray | None = None
    total_weight: float = 0.0

    def build_distribution(self) -> None:
        """BuildEnvironmentDistribution (src/lighting/environment.cpp:73-123)."""
        h, w = self.texels.shape[:2]
        self.texels = np.ascontiguousarray(self.texels, np.float32)
        tw = np.zeros(h * w, np.float32)
        rw = np.zeros(h, np.float32)
        rc = np.zeros(h, np.float32)
        cc = np.zeros(h * w, np.float32)
        tot = C.c_float()
        check(_bind().yrc_environment_distribution_build(ptr(self.texels), w, h, ptr(tw), ptr(rw), ptr(rc),
                                                         ptr(cc), C.byref(tot)))
        self.texel_weights, self.row_weights, self.row_cdf, self.conditional_cdfs = tw, rw, rc, cc
        self.total_weight = float(tot.value)


def build_bssrdf_table(eta: float, g: float = 0.0, rho_count: int = 100, radius_count: int = 64) -> dict:
    """ComputeBeamDiffusionBSSRDF (src/shading/bssrdf.cpp:124-151): the
    profile table a subsurface material with relative index `eta` uses (the
    reference's compiler builds 100 x 64 with g = 0)."""
    t = {"rho_samples": np.zeros(rho_count, np.float32), "radius_samples": np.zeros(radius_count, np.float32),
         "profile": np.zeros(rho_count * radius_count, np.float32), "rho_eff": np.zeros(rho_count, np.float32),
         "profile_cdf": np.zeros(rho_count * radius_count, np.float32)}
    check(_bind().yrc_bssrdf_table_build(g, eta, rho_count, radius_count, ptr(t["rho_samples"]),
                                         ptr(t["radius_samples"]), ptr(t["profile"]), ptr(t["rho_eff"]),
                                         ptr(t["profile_cdf"])))
    return t


def build_alias_table(weights: np.ndarray):
    """BuildAliasTable (src/lighting/light_sampling.cpp:148-183)."""
    w = np.ascontiguousarray(weights, np.float32)
    n = w.size
    prob = np.zeros(n, np.float32)
    alias = np.zeros(n, np.int32)
    pmf = np.zeros(n, np.float32)
    check(_bind().yrc_alias_table_build(ptr(w), n, ptr(prob), ptr(alias), ptr(pmf)))
    return prob, alias, pmf


@dataclass
class RenderScene:
    """RenderSceneIR + RenderSettings as numpy arrays."""

    geometry: SceneGeometry
    materials: np.ndarray                      # MATERIAL_DTYPE
    camera: dict                               # origin, forward, right, up, fov_y_radians
    width: int
    height: int
    spp: int = 1
    max_depth: int = 5
    seed: int = 0
    sampler: int = INDEPENDENT
    radiance_clamp: float = 0.0
    normals: np.ndarray | None = None          # (V, 3) shading normals
    emissive: np.ndarray = field(default_factory=lambda: np.zeros(0, EMISSIVE_DTYPE))
    alias: tuple | None = None                 # (probability, alias, pmf) over emissive power
    environment: EnvironmentMap = field(default_factory=EnvironmentMap)
    bssrdf_tables: list = field(default_factory=list)  # build_bssrdf_table() dicts, by bssrdf_index
    adaptive: dict | None = None               # enabled/min_spp/relative_error/absolute_error/confidence
    uvs: np.ndarray | None = None              # (V, 2) RenderVertex::uv
    tangents: np.ndarray | None = None         # (V, 4) RenderVertex::tangent xyz + tangent_handedness
    textures: list = field(default_factory=list)  # texture.Texture, by material texture index
    measured: list = field(default_factory=list)  # measured.MeasuredBrdf, by material measured_index
    analytic: np.ndarray = field(default_factory=lambda: np.zeros(0, ANALYTIC_DTYPE))  # point/spot/distant lights

    def emissive_power_alias(self):
        """The alias table PrepareLightSampling builds (emissive power = area * luminance)."""
        if self.alias is None:
            rad = self.emissive["radiance"].astype(np.float32)
            lum = np.maximum(np.float32(0), np.float32(0.2126) * rad[:, 0] + np.float32(0.7152) * rad[:, 1]
                             + np.float32(0.0722) * rad[:, 2]).astype(np.float32)
            area = self.emissive["area"].astype(np.float32)
            area = np.where(np.isfinite(area) & (area > 0), area, np.float32(0)).astype(np.float32)
            self.alias = build_alias_table((area * lum).astype(np.float32))
        return self.alias


@dataclass
class RenderResult:
    """RenderResult (backend.hpp:57-62): ok/error, the film, stats."""

    ok: bool
    error: str = ""
    film: np.ndarray | None = None             # FILM_PIXEL_DTYPE, (H, W)
    bad_samples: int = 0
    stats: dict = field(default_factory=dict)

    def linear(self) -> np.ndarray:
        """Film::LinearPixel for every pixel: (H, W, 3) float32."""
        s = self.film["samples"].astype(np.float32)
        out = np.zeros(self.film["sum"].shape, np.float32)
        nz = s > 0
        out[nz] = self.film["sum"][nz] / s[nz][:, None]
        return out


def scene_desc(scene: RenderScene, accel=None):
    """The C-ABI yrc_scene_desc of `scene` (and the arrays it points into,
    which the caller must keep alive while the descriptor is used)."""
    holder = type("DescHolder", (), {})()
    PreparedScene._fill(holder, scene, accel)
    return holder._desc, holder


class PreparedScene:
    """CudaPreparedScene: the scene resident in HBM (yrc_render_scene)."""

    def __init__(self, scene: RenderScene, accel):
        L = _bind()
        PreparedScene._fill(self, scene, accel)
        self._handle = C.c_void_p()
        check(L.yrc_render_scene_create(C.byref(self._desc), C.byref(self._handle)))

    @staticmethod
    def _fill(self, scene: RenderScene, accel) -> None:
        self.scene = scene
        self._keep = []
        d = SceneDesc()
        d.geometry = scene.geometry.c_struct()
        if scene.normals is not None:
            nrm = np.ascontiguousarray(scene.normals, np.float32).reshape(-1, 3)
            self._keep.append(nrm)
            d.normals = ptr(nrm)
            d.normal_stride = 12
        if scene.uvs is not None:
            uv = np.ascontiguousarray(scene.uvs, np.float32).reshape(-1, 2)
            self._keep.append(uv)
            d.uvs = ptr(uv)
            d.uv_stride = 8
        if scene.tangents is not None:
            tg = np.ascontiguousarray(scene.tangents, np.float32).reshape(-1, 4)
            self._keep.append(tg)
            d.tangents = ptr(tg)
            d.tangent_stride = 16
        if scene.textures:
            tarr, tkeep = textures_array(scene.textures)
            self._keep += [tarr, tkeep]
            d.textures = C.addressof(tarr)
            d.texture_count = len(scene.textures)
        if scene.measured:
            marr, mkeep = measured_array(scene.measured)
            self._keep += [marr, mkeep]
            d.measured = C.addressof(marr)
            d.measured_count = len(scene.measured)
        if scene.analytic.size:
            an = np.ascontiguousarray(scene.analytic, ANALYTIC_DTYPE)
            self._keep.append(an)
            d.analytic = ptr(an)
            d.analytic_count = an.size  # the power alias table is built by the library
        mats = np.ascontiguousarray(scene.materials, MATERIAL_DTYPE)
        em = np.ascontiguousarray(scene.emissive, EMISSIVE_DTYPE)
        self._keep += [mats, em]
        d.materials = ptr(mats)
        d.material_count = mats.size
        d.emissive = ptr(em)
        d.emissive_count = em.size
        if em.size:
            prob, alias, pmf = [np.ascontiguousarray(a) for a in scene.emissive_power_alias()]
            self._keep += [prob, alias, pmf]
            d.emissive_power = AliasTable(ptr(prob), ptr(alias), ptr(pmf), em.size)
        env = scene.environment
        e = Environment()
        e.active = int(env.active)
        e.radiance[:] = [float(x) for x in env.radiance]
        e.strength = env.strength
        e.rotation_radians = env.rotation
        if env.active and env.texels is not None:
            if env.texel_weights is None:
                env.build_distribution()
            tex = np.ascontiguousarray(env.texels, np.float32)
            self._keep += [tex, env.texel_weights, env.row_weights, env.row_cdf, env.conditional_cdfs]
            e.height, e.width = tex.shape[:2]
            e.texels = ptr(tex)
            e.texel_weights = ptr(env.texel_weights)
            e.row_weights = ptr(env.row_weights)
            e.row_cdf = ptr(env.row_cdf)
            e.conditional_cdfs = ptr(env.conditional_cdfs)
            e.total_weight = env.total_weight
        d.environment = e
        if scene.bssrdf_tables:
            tabs = (BssrdfTable * len(scene.bssrdf_tables))()
            for i, t in enumerate(scene.bssrdf_tables):
                arrays = {k: np.ascontiguousarray(v, np.float32) for k, v in t.items()}
                self._keep.append(arrays)
                tabs[i] = BssrdfTable(arrays["rho_samples"].size, arrays["radius_samples"].size,
                                      ptr(arrays["rho_samples"]), ptr(arrays["radius_samples"]),
                                      ptr(arrays["profile"]), ptr(arrays["rho_eff"]), ptr(arrays["profile_cdf"]))
            self._keep.append(tabs)
            d.bssrdf_tables = C.addressof(tabs)
            d.bssrdf_count = len(scene.bssrdf_tables)
        cam = scene.camera
        d.camera = Camera((C.c_float * 3)(*cam["origin"]), (C.c_float * 3)(*cam["forward"]),
                          (C.c_float * 3)(*cam["right"]), (C.c_float * 3)(*cam["up"]), cam["fov_y_radians"])
        ad = scene.adaptive or {}
        d.settings = Settings(scene.width, scene.height, scene.spp, scene.max_depth, scene.seed, scene.sampler,
                              scene.radiance_clamp, int(ad.get("enabled", False)), int(ad.get("min_spp", 16)),
                              float(ad.get("relative_error", 0.05)), float(ad.get("absolute_error", 0.001)),
                              float(ad.get("confidence", 1.96)))
        if accel is not None and hasattr(accel, "blases"):
            tv, keep = accel.view()
            self._keep.append(keep)
            self._tv = tv
            d.two_level = C.addressof(tv)
        elif accel is not None:
            bv = accel.view()
            self._bv = bv
            d.flat = C.addressof(bv)
        self._desc = d

    @property
    def device_bytes(self) -> int:
        return int(_bind().yrc_render_scene_device_bytes(self._handle))

    @property
    def capacity(self) -> int:
        """Paths in flight per batch (queue capacity) of the next render."""
        return int(_bind().yrc_render_scene_capacity(self._handle))

    def set_capacity(self, capacity: int) -> None:
        """Sets the queue capacity (0 restores the default); bounded to whole
        passes of the image. The film does not depend on it."""
        check(_bind().yrc_render_scene_set_capacity(self._handle, int(capacity)))

    def autotune(self, capacity: bool = True, trace_shape: bool = True) -> dict:
        """Times probe renders of this scene for each candidate queue
        capacity and traversal launch shape and keeps the fastest."""
        t = RenderTuning()
        flags = (TUNE_CAPACITY if capacity else 0) | (TUNE_TRACE_SHAPE if trace_shape else 0)
        check(_bind().yrc_render_autotune(self._handle, flags, C.byref(t)))
        return {"capacity": int(t.capacity), "trace_shape": int(t.trace_shape), "candidates": int(t.candidates),
                "seconds_per_sample": float(t.seconds_per_sample)}

    def set_tuning(self, tuning: dict) -> None:
        """Applies an autotune() result (capacity and traversal launch shape),
        e.g. one found on a scene of the same image size and spp."""
        t = RenderTuning(int(tuning["capacity"]), int(tuning["trace_shape"]), 0, 0.0)
        check(_bind().yrc_render_scene_set_tuning(self._handle, C.byref(t)))

    def set_view(self, camera: dict, seed: int) -> None:
        """A new camera (origin, forward, right, up, fov_y_radians) and
        sampler seed for the next render; the scene's working memory and
        captured batch are kept."""
        cam = Camera()
        for k in ("origin", "forward", "right", "up"):
            getattr(cam, k)[:] = [float(x) for x in camera[k]]
        cam.fov_y_radians = float(camera["fov_y_radians"])
        check(_bind().yrc_render_scene_set_view(self._handle, C.byref(cam), C.c_uint64(seed)))
        self.scene = dataclasses.replace(self.scene, camera=dict(camera), seed=int(seed))

    def shadow_visibility(self, rays: np.ndarray) -> np.ndarray:
        """TraceShadowVisibility through this scene's shadow stage for (n, 8)
        rays (origin, t_min, direction, max_distance) -> (n, 4): RGB
        transmittance and 1 when visible, all 0 when occluded."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        out = np.empty((r.shape[0], 4), np.float32)
        check(_bind().yrc_render_scene_shadow_eval(self._handle, ptr(r), r.shape[0], ptr(out)))
        return out

    def set_radiance_cache(self, cache, spread_threshold: float = 0.01, train_one_in: int = 16,
                           train_records: int = 65536, train: bool = True, train_steps: int = 1,
                           delta_vertices: bool = False, averaged: bool = False) -> None:
        """Attaches a yaoray_b200.nrc.RadianceCache (None detaches): paths end
        at the cache when their footprint heuristic fires, and the cache
        takes `train_steps` optimiser steps per batch on the records of 1 in
        `train_one_in` unbiased paths. With `delta_vertices` a path may also
        end at a specular (delta) vertex once its spread is large; with
        `averaged` the paths query the moving average of the cache's
        parameters instead of the latest ones."""
        st = CacheSettings(spread_threshold, train_one_in, train_records, 1 if train else 0, train_steps,
                           1 if delta_vertices else 0, 1 if averaged else 0)
        self._cache = cache
        check(_bind().yrc_render_scene_set_cache(self._handle, cache._handle if cache is not None else None,
                                                 C.byref(st)))

    def close(self):
        if getattr(self, "_handle", None) and self._handle.value:
            _bind().yrc_render_scene_destroy(self._handle)
            self._handle = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


@dataclass
class RenderRequestPy:
    """RenderRequest (backend.hpp:33-38)."""

    resume_film: np.ndarray | None = None
    resume_completed_spp: int = 0
    resume_bad_samples: int = 0
    stop: object | None = None                 # ctypes c_int32: non-zero cancels
    progress_callback: object | None = None    # f(progress dict, film) -> (cancel, error)


def pinned_film(width: int, height: int) -> np.ndarray:
    """A (height, width) FILM_PIXEL_DTYPE array in pinned host memory, for
    CudaBackend.render(..., film_out=...): the film's device-to-host copy
    then runs at full link speed and touches no fresh pages."""
    import torch

    buf = torch.empty(width * height * FILM_PIXEL_DTYPE.itemsize, dtype=torch.uint8).pin_memory()
    return buf.numpy().view(FILM_PIXEL_DTYPE).reshape(height, width)


class CudaBackend:
    """RenderBackend for RenderBackendKind::Cuda over libyrcuda."""

    def kind(self) -> str:
        return "cuda"

    def capabilities(self) -> dict:
        return {"kind": "cuda", "runnable": True, "supports_debug_direct": False, "supports_path": True,
                "supports_offline_progress": True, "supports_texture_materials": False}

    def prepare(self, scene: RenderScene, accel=None) -> PreparedScene:
        """Builds the reference-layout BVH on the device (unless given; the
        reference's bytes, see accel.build_bvh_device) and uploads."""
        if accel is None:
            if scene.geometry.instances.size:
                accel = build_two_level_bvh(scene.geometry, device=True)
            else:
                accel = build_bvh_device(scene.geometry)[0]
        return PreparedScene(scene, accel)

    def render(self, prepared: PreparedScene, request: RenderRequestPy | None = None,
               film_out: np.ndarray | None = None) -> RenderResult:
        """CudaBackend::Render. `film_out` (optional) is a caller-owned
        (height, width) FILM_PIXEL_DTYPE array that receives the film, e.g. a
        pinned buffer kept across the frames of an interactive renderer
        (the copy into pinned memory is direct; a fresh array is allocated
        and page-faulted in on every call otherwise)."""
        L = _bind()
        sc = prepared.scene
        req = request or RenderRequestPy()
        r = Request()
        keep = []
        if req.resume_film is not None:
            rf = np.ascontiguousarray(req.resume_film, FILM_PIXEL_DTYPE).reshape(-1)
            keep.append(rf)
            r.resume_film = ptr(rf)
        r.resume_completed_spp = req.resume_completed_spp
        r.resume_bad_samples = req.resume_bad_samples
        if req.stop is not None:
            r.stop_flag = C.addressof(req.stop)
        if req.progress_callback is not None:
            def cb(p, film_ptr, bad, user, err, cap):
                film = np.frombuffer((C.c_char * (sc.width * sc.height * 56)).from_address(film_ptr),
                                     FILM_PIXEL_DTYPE).reshape(sc.height, sc.width).copy()
                prog = {f[0]: getattr(p.contents, f[0]) for f in Progress._fields_}
                cancel, msg = req.progress_callback(prog, film)
                if cancel and msg and err and cap > 0:
                    data = msg.encode()[: cap - 1] + b"\0"
                    C.memmove(err, data, len(data))
                return 1 if cancel else 0
            r.progress = PROGRESS_FN(cb)
            keep.append(r.progress)
        if film_out is not None:
            if (film_out.dtype != FILM_PIXEL_DTYPE or film_out.shape != (sc.height, sc.width)
                    or not film_out.flags.c_contiguous):
                raise ValueError("film_out must be a C-contiguous (height, width) FILM_PIXEL_DTYPE array")
            film = film_out
        else:
            film = np.zeros((sc.height, sc.width), FILM_PIXEL_DTYPE)
        bad = C.c_uint64()
        st = Stats()
        status = L.yrc_render(prepared._handle, C.byref(r), ptr(film), C.byref(bad), C.byref(st))
        if status != _lib.YRC_OK:
            msg = L.yrc_last_error().decode(errors="replace")
            if status in (_lib.YRC_ERR_CANCELLED, _lib.YRC_ERR_INVALID_ARGUMENT):
                return RenderResult(False, msg)
            raise YrcError(status, msg)
        stats = {f[0]: getattr(st, f[0]) for f in Stats._fields_}
        return RenderResult(True, "", film, int(bad.value), stats)

    def render_many(self, prepared: list, pooled: bool = False) -> list:
        """Renders several prepared scenes together (yrc_render_many): each
        step is one launch of a graph holding every unfinished scene's batch.
        With `pooled` (yrc_render_pooled), each bounce traces the extend and
        shadow rays of all scenes in one persistent launch each. Films equal
        render()'s; stats["device_seconds"] is the whole call's."""
        L = _bind()
        n = len(prepared)
        if n == 0:
            return []
        films = [np.zeros((p.scene.height, p.scene.width), FILM_PIXEL_DTYPE) for p in prepared]
        handles = (C.c_void_p * n)(*[p._handle.value for p in prepared])
        film_ptrs = (C.c_void_p * n)(*[f.ctypes.data for f in films])
        bads = (C.c_uint64 * n)()
        stats = (Stats * n)()
        secs = C.c_double()
        call = L.yrc_render_pooled if pooled else L.yrc_render_many
        status = call(handles, n, None, film_ptrs, bads, stats, C.byref(secs))
        if status != _lib.YRC_OK:
            msg = L.yrc_last_error().decode(errors="replace")
            if status in (_lib.YRC_ERR_CANCELLED, _lib.YRC_ERR_INVALID_ARGUMENT):
                return [RenderResult(False, msg) for _ in prepared]
            raise YrcError(status, msg)
        return [RenderResult(True, "", films[i], int(bads[i]), {f[0]: getattr(stats[i], f[0]) for f in Stats._fields_})
                for i in range(n)]
