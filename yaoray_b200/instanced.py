"""Instanced scene of the batched wavefront configuration: a two-level BVH of
256 random affine instances of four procedural meshes — three displaced tori
(50,000, 75,000 and 100,000 triangles) and a heightfield (249,218 triangles),
≈30M instanced triangles — over a ground plane.

Materials are drawn per instanced object: 40 % Lambertian (albedo
U[0.1, 0.8]), 25 % GGX conductor (alpha U[0.05, 0.5], gold-like RGB eta/k,
carried as reflectance = ConductorF0(eta, k) because the reference's plain
conductor is Schlick on `reflectance`),
20 % rough dielectric (eta 1.5), 15 % coated diffuse (dielectric coat,
thickness 0.01, Beer–Lambert absorption U[0, 0.5]). Lights: a procedural
2048 x 1024 FP32 HDRI (sky gradient plus a 0.5 degree sun disk of radiance
1e4, importance-sampled through the environment distribution) and 64 emissive
triangles in the emissive-power alias table. Render: 1920 x 1080, 256 spp
Owen-scrambled Sobol (seed 0), max depth 16, RGB FP32 film.

The scene is built directly as a RenderSceneIR in the layout the reference
compiles ObjectBegin/ObjectInstance files into
(src/frontend/pbrt/scene_compiler_geometry.cpp:62-126): every
(mesh, material) object is one primitive referenced by its instances, and
every primitive that no instance references (ground plane, emitters) gets an
identity instance after the others. Objects of one mesh share its vertices but
own their index ranges, so each flat triangle index belongs to one primitive.

`scene(..., mesh_scale=s, instances=n, env_width=w)` shrinks the meshes
(triangle counts × s), the instance count and the HDRI for parity tests that
the reference CPU backend finishes in seconds.
"""
from __future__ import annotations

import math

import numpy as np

from . import _lib
from .accel import SceneGeometry
from .render import (COATED_DIFFUSE, CONDUCTOR, DIELECTRIC, DIFFUSE, EMISSIVE_DTYPE, OWEN_SOBOL, EnvironmentMap,
                     RenderScene, default_material)

WIDTH, HEIGHT, SPP, MAX_DEPTH = 1920, 1080, 256, 16
INSTANCES = 256
OBJECTS = 32                      # (mesh, material) pairs, 8 per mesh
EMITTERS = 64
# Gold, RGB approximation of its complex index of refraction.
GOLD_ETA = (0.143, 0.374, 1.442)
GOLD_K = (3.983, 2.385, 1.603)


def conductor_f0(eta: float, k: float) -> float:
    """ConductorF0 (scene_compiler_conductor_materials.cpp:116-120), in float32."""
    e, kk = np.float32(eta), np.float32(k)
    num = (e - np.float32(1)) * (e - np.float32(1)) + kk * kk
    den = (e + np.float32(1)) * (e + np.float32(1)) + kk * kk
    return float(num / den) if den > 0 else 1.0


GOLD_F0 = tuple(conductor_f0(e, k) for e, k in zip(GOLD_ETA, GOLD_K))
SUN_RADIANCE = 1.0e4
SUN_DIAMETER_DEG = 0.5
EYE = (0.0, 55.0, -150.0)
LOOK = (0.0, 12.0, 0.0)
FOV = 40.0

# (kind, tori grid (nu, nv) or heightfield cells (nx, nz)), full size.
MESHES = (("torus", 250, 100), ("torus", 250, 150), ("torus", 250, 200), ("heightfield", 353, 353))


def _vertex_normals(p: np.ndarray, t: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals (float32, unit length)."""
    a, b, c = p[t[:, 0]], p[t[:, 1]], p[t[:, 2]]
    fn = np.cross(b - a, c - a)
    n = np.zeros_like(p, dtype=np.float64)
    for k in range(3):
        for axis in range(3):
            n[:, axis] += np.bincount(t[:, k], weights=fn[:, axis], minlength=p.shape[0])
    length = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.where(length > 0, n / np.maximum(length, 1e-30), np.array([0.0, 1.0, 0.0]))
    return n.astype(np.float32)


def displaced_torus(nu: int, nv: int, major: float, minor: float, amp: float, ku: int, kv: int):
    """Torus around +y with its tube radius modulated by two sine products;
    2 * nu * nv triangles wound outward."""
    u = 2.0 * np.pi * np.arange(nu) / nu
    v = 2.0 * np.pi * np.arange(nv) / nv
    uu, vv = np.meshgrid(u, v, indexing="ij")
    r = minor * (1.0 + amp * np.sin(ku * uu) * np.cos(kv * vv) + 0.5 * amp * np.sin(3 * ku * uu + 2 * kv * vv))
    ring = major + r * np.cos(vv)
    p = np.stack([ring * np.cos(uu), r * np.sin(vv), ring * np.sin(uu)], -1).reshape(-1, 3)
    i = np.arange(nu)[:, None]
    j = np.arange(nv)[None, :]
    a = i * nv + j
    b = ((i + 1) % nu) * nv + j
    c = ((i + 1) % nu) * nv + (j + 1) % nv
    d = i * nv + (j + 1) % nv
    tris = np.concatenate([np.stack([a, c, b], -1).reshape(-1, 3), np.stack([a, d, c], -1).reshape(-1, 3)])
    return p.astype(np.float32), tris.astype(np.uint32)


def heightfield(nx: int, nz: int, size: float, height: float, rng: np.random.Generator):
    """Square sheet of nx * nz cells (2 triangles each, facing +y) displaced by
    a sum of sines and Gaussian bumps."""
    x = np.linspace(-size / 2, size / 2, nx + 1)
    z = np.linspace(-size / 2, size / 2, nz + 1)
    xx, zz = np.meshgrid(x, z, indexing="ij")
    h = 0.25 * np.sin(1.7 * xx / size * 2 * np.pi) * np.cos(2.3 * zz / size * 2 * np.pi)
    for _ in range(6):
        cx, cz = rng.uniform(-size / 3, size / 3, 2)
        w = rng.uniform(0.08, 0.2) * size
        h += rng.uniform(0.3, 1.0) * np.exp(-((xx - cx) ** 2 + (zz - cz) ** 2) / (2 * w * w))
    p = np.stack([xx, height * h, zz], -1).reshape(-1, 3)
    i = np.arange(nx)[:, None]
    j = np.arange(nz)[None, :]
    a = i * (nz + 1) + j
    b = (i + 1) * (nz + 1) + j
    c = (i + 1) * (nz + 1) + j + 1
    d = i * (nz + 1) + j + 1
    tris = np.concatenate([np.stack([a, c, b], -1).reshape(-1, 3), np.stack([a, d, c], -1).reshape(-1, 3)])
    return p.astype(np.float32), tris.astype(np.uint32)


def meshes(mesh_scale: float = 1.0, seed: int = 11):
    """The four procedural meshes as [(positions, triangles, normals)]."""
    rng = np.random.default_rng(seed)
    f = math.sqrt(mesh_scale)
    out = []
    for k, (kind, n0, n1) in enumerate(MESHES):
        a, b = max(6, round(n0 * f)), max(4, round(n1 * f))
        if kind == "torus":
            p, t = displaced_torus(a, b, major=4.0 + k, minor=1.2 + 0.3 * k, amp=0.18, ku=5 + 2 * k, kv=3 + k)
        else:
            p, t = heightfield(a, b, size=14.0, height=4.0, rng=rng)
        out.append((p, t, _vertex_normals(p, t)))
    return out


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    x, y, z, w = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _affine(rng: np.random.Generator, spread: float) -> np.ndarray:
    """Column-major Mat4f (TransformPoint reads m[0], m[4], m[8], m[12] for x)
    of translate * rotate * shear * scale; x and z within +-95 * spread."""
    s = np.diag(rng.uniform(0.6, 1.4, 3))
    shear = np.eye(3)
    shear[0, 1], shear[2, 1] = rng.uniform(-0.25, 0.25, 2)
    m = np.eye(4)
    m[:3, :3] = _random_rotation(rng) @ shear @ s
    m[:3, 3] = (spread * rng.uniform(-95.0, 95.0), rng.uniform(3.0, 14.0), spread * rng.uniform(-95.0, 95.0))
    return m.T.reshape(16).astype(np.float32)


def materials(rng: np.random.Generator) -> np.ndarray:
    """The OBJECTS-entry palette: 13 Lambertian, 8 conductor, 6 rough
    dielectric, 5 coated diffuse (40/25/19/16 % of the objects), shuffled."""
    kinds = [DIFFUSE] * 13 + [CONDUCTOR] * 8 + [DIELECTRIC] * 6 + [COATED_DIFFUSE] * 5
    rng.shuffle(kinds)
    out = []
    for kind in kinds:
        if kind == DIFFUSE:
            out.append(default_material(reflectance=rng.uniform(0.1, 0.8, 3)))
        elif kind == CONDUCTOR:
            # The reference's plain conductor shades with Schlick on
            # `reflectance` and ignores eta/k, so the gold colour is carried
            # as ConductorF0(eta, k) per channel
            # (src/frontend/pbrt/scene_compiler_conductor_materials.cpp:116-120).
            alpha = rng.uniform(0.05, 0.5)
            out.append(default_material(kind=CONDUCTOR, eta=GOLD_ETA, k=GOLD_K, reflectance=GOLD_F0,
                                        uroughness=alpha, vroughness=alpha, remap_roughness=0))
        elif kind == DIELECTRIC:
            alpha = rng.uniform(0.05, 0.3)
            out.append(default_material(kind=DIELECTRIC, ior=1.5, uroughness=alpha, vroughness=alpha,
                                        remap_roughness=0))
        else:
            out.append(default_material(kind=COATED_DIFFUSE, reflectance=rng.uniform(0.1, 0.8, 3), coating_ior=1.5,
                                        coating_roughness=0.0, coat_thickness=0.01,
                                        coat_absorption=rng.uniform(0.0, 0.5, 3)))
    return np.stack(out)


def sun_direction() -> np.ndarray:
    elev, azim = math.radians(38.0), math.radians(-35.0)
    return np.array([math.cos(elev) * math.sin(azim), math.sin(elev), math.cos(elev) * math.cos(azim)])


def hdri(width: int = 2048, height: int = 1024) -> np.ndarray:
    """RGBA32F equirectangular sky in the reference's mapping
    (DirectionToEnvironmentUv, src/lighting/environment.cpp:54-60: +y up,
    row 0 at the zenith, u = 0.5 + atan2(x, z) / 2pi): a gradient from a
    blue zenith to a pale horizon, a dark ground below it, and a sun disk of
    diameter 0.5 degree with radiance 1e4. Texels the disk touches blend sky
    and sun by the fraction of the texel the disk covers (32 x 32 sub-samples),
    so the sun keeps its power at any map resolution."""
    def directions(theta, phi):
        return np.stack([np.sin(theta) * np.sin(phi), np.cos(theta), np.sin(theta) * np.cos(phi)], -1)

    def sky(d):
        up = np.clip(d[..., 1], 0.0, 1.0)[..., None]
        zenith = np.array([0.25, 0.45, 1.0])
        horizon = np.array([1.0, 0.95, 0.85])
        return np.where(d[..., 1:2] >= 0.0, horizon + (zenith - horizon) * np.sqrt(up), np.array([0.12, 0.11, 0.10]))

    theta = (np.arange(height) + 0.5) * np.pi / height
    phi = ((np.arange(width) + 0.5) / width - 0.5) * 2 * np.pi
    th, ph = np.meshgrid(theta, phi, indexing="ij")
    rgb = sky(directions(th, ph))
    sun = sun_direction()
    cos_disk = math.cos(math.radians(SUN_DIAMETER_DEG / 2))
    # Candidate texels: rows/columns around the sun's texel.
    s_theta = math.acos(sun[1])
    s_phi = math.atan2(sun[0], sun[2])
    row = int(s_theta / math.pi * height)
    col = int((s_phi / (2 * math.pi) + 0.5) * width) % width
    reach = 2 + int(math.radians(SUN_DIAMETER_DEG) / min(math.pi / height, 2 * math.pi / width) / max(
        math.sin(s_theta), 1e-3))
    sub = (np.arange(32) + 0.5) / 32
    for y in range(max(0, row - reach), min(height, row + reach + 1)):
        for xx in range(col - reach, col + reach + 1):
            x = xx % width
            t = (y + sub[:, None]) * np.pi / height
            p = ((x + sub[None, :]) / width - 0.5) * 2 * np.pi
            d = directions(np.broadcast_to(t, (32, 32)), np.broadcast_to(p, (32, 32)))
            inside = d @ sun >= cos_disk
            if inside.any():
                f = inside.mean()
                rgb[y, x] = (1 - f) * rgb[y, x] + f * SUN_RADIANCE
    tex = np.ones((height, width, 4), np.float32)
    tex[..., :3] = rgb
    return tex


def camera(spread: float = 1.0, orbit: float = 0.0) -> dict:
    """The pinhole camera; `orbit` (radians) turns the eye about the vertical
    axis through the look-at point (a camera orbit; 0 is the default view)."""
    eye = np.array(EYE, np.float32) * np.float32(spread)
    look = np.array(LOOK, np.float32) * np.float32(spread)
    if orbit:
        c, s = np.float32(math.cos(orbit)), np.float32(math.sin(orbit))
        rel = eye - look
        eye = (look + np.array([c * rel[0] + s * rel[2], rel[1], -s * rel[0] + c * rel[2]], np.float32)).astype(np.float32)
    fwd = look - eye
    fwd = fwd / np.float32(np.sqrt(np.float32(np.dot(fwd, fwd))))
    right = np.cross(fwd, np.array([0, 1, 0], np.float32)).astype(np.float32)
    right = right / np.float32(np.sqrt(np.float32(np.dot(right, right))))
    up = np.cross(right, fwd).astype(np.float32)
    return {"origin": tuple(map(float, eye)), "forward": tuple(map(float, fwd)), "right": tuple(map(float, right)),
            "up": tuple(map(float, up)), "fov_y_radians": float(np.float32(FOV) * np.float32(math.pi) / np.float32(180))}


def _triangle_area(a, b, c) -> np.float32:
    cr = np.cross((b - a).astype(np.float32), (c - a).astype(np.float32)).astype(np.float32)
    return np.float32(np.float32(np.sqrt(np.float32(np.dot(cr, cr)))) * np.float32(0.5))


def scene(width: int = WIDTH, height: int = HEIGHT, spp: int = SPP, max_depth: int = MAX_DEPTH,
          instances: int = INSTANCES, mesh_scale: float = 1.0, env_width: int = 2048, seed: int = 5) -> RenderScene:
    rng = np.random.default_rng(seed)
    # Fewer instances are packed closer (same density), with the camera and
    # the emitters' x/z pulled in by the same factor.
    spread = max(0.25, math.sqrt(instances / INSTANCES))
    mesh_list = meshes(mesh_scale)
    palette = materials(rng)

    pos, nrm, idx, prims = [], [], [], []
    vbase = ibase = 0
    mesh_vbase = []
    for p, t, n in mesh_list:
        pos.append(p)
        nrm.append(n)
        mesh_vbase.append(vbase)
        vbase += p.shape[0]
    # One primitive per (mesh, material) object; objects of a mesh share its
    # vertices and own an index range.
    for o in range(OBJECTS):
        m = o % len(mesh_list)
        t = mesh_list[m][1]
        idx.append((t + mesh_vbase[m]).reshape(-1))
        prims.append((ibase, t.size, o, 1))
        ibase += t.size
    mats = [palette[o] for o in range(OBJECTS)]

    # Ground plane (y = 0, facing +y).
    g = 160.0
    ground_p = np.array([[-g, 0, -g], [-g, 0, g], [g, 0, g], [g, 0, -g]], np.float32)
    ground_t = np.array([[0, 1, 2], [0, 2, 3]], np.uint32)
    pos.append(ground_p)
    nrm.append(np.tile(np.array([[0, 1, 0]], np.float32), (4, 1)))
    idx.append((ground_t + vbase).reshape(-1))
    mats.append(default_material(reflectance=(0.5, 0.5, 0.5)))
    prims.append((ibase, 6, len(mats) - 1, 0))
    vbase += 4
    ibase += 6

    # 64 emissive triangles facing down, each its own primitive and material.
    emissive = np.zeros(EMITTERS, EMISSIVE_DTYPE)
    for e in range(EMITTERS):
        c = np.array([spread * rng.uniform(-85, 85), rng.uniform(22, 45), spread * rng.uniform(-85, 85)])
        size = rng.uniform(1.5, 3.5)
        ang = rng.uniform(0, 2 * np.pi)
        corners = [c + size * np.array([math.cos(ang + k * 2 * np.pi / 3), rng.uniform(-0.2, 0.2),
                                        math.sin(ang + k * 2 * np.pi / 3)]) for k in range(3)]
        tri = np.array(corners, np.float32)
        if np.cross(tri[1] - tri[0], tri[2] - tri[0])[1] > 0:  # face down
            tri = tri[[0, 2, 1]]
        radiance = rng.uniform(0.4, 1.0, 3) * rng.uniform(8.0, 40.0)
        pos.append(tri)
        nrm.append(np.zeros((3, 3), np.float32))
        idx.append(np.arange(3, dtype=np.uint32) + vbase)
        mats.append(default_material(reflectance=(0.5, 0.5, 0.5), emission=radiance))
        prims.append((ibase, 3, len(mats) - 1, 0))
        emissive[e]["primitive_index"] = len(prims) - 1
        emissive[e]["radiance"] = radiance
        emissive[e]["area"] = _triangle_area(tri[0], tri[1], tri[2])
        vbase += 3
        ibase += 3

    inst = np.zeros(instances + len(prims) - OBJECTS, _lib.INSTANCE_DTYPE)
    for k in range(instances):
        inst[k]["primitive"] = rng.integers(OBJECTS)
        inst[k]["object_to_world"] = _affine(rng, spread)
    ident = np.eye(4, dtype=np.float32).reshape(16)
    for k, prim in enumerate(range(OBJECTS, len(prims))):
        inst[instances + k]["primitive"] = prim
        inst[instances + k]["object_to_world"] = ident

    geom = SceneGeometry(np.concatenate(pos), np.concatenate(idx), np.array(prims, dtype=_lib.PRIM_DTYPE),
                         instances=inst)
    env_height = env_width // 2
    env = EnvironmentMap(active=True, radiance=(1.0, 1.0, 1.0), strength=1.0, rotation=0.0,
                         texels=hdri(env_width, env_height))
    env.build_distribution()
    return RenderScene(geom, np.stack(mats), camera(spread), width, height, spp=spp, max_depth=max_depth, seed=0,
                       sampler=OWEN_SOBOL, normals=np.concatenate(nrm), emissive=emissive, environment=env)


def instanced_triangles(s: RenderScene) -> int:
    """Triangles summed over all instances (each instance counts its
    primitive's triangles)."""
    per_prim = s.geometry.primitives["index_count"] // 3
    return int(per_prim[s.geometry.instances["primitive"]].sum())
