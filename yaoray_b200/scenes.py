"""Seeded synthetic scenes and ray sets with the shapes of the benchmark
workloads (no external datasets exist for them; every input is generated).

Traversal set ("2M triangles"): 512 noisy spheres of 4096 triangles each =
2,097,152 FP32 triangles inside a 100^3 box. 4096 is not an icosphere count
(20 * 4^k), so each sphere is a latitude-longitude tessellation with 64
slices and 33 stacks whose pole stacks are triangle fans:
64 + 64 + 31 * 64 * 2 = 4096 non-degenerate triangles. Radius U[0.5, 3],
per-vertex radial noise U[-5%, +5%], a uniformly random rotation, centre
U[0, 100]^3. One RenderPrimitive per sphere.

Ray sets (7,997,584 = 2828^2 rays each at full size):
  coherent   — pinhole camera primary rays through pixel centres, camera at
               (50, 50, 190) looking down -z with a 40 degree vertical fov;
  incoherent — origin U[box], direction uniform on the sphere;
  shadow     — origin U[box] towards a uniform random point in the box,
               t_max = the distance to that point (any-hit queries).
Rays are (N, 8) float32 rows: origin.xyz, t_min, direction.xyz, t_max.
"""
from __future__ import annotations

import numpy as np

from .accel import SceneGeometry

RAY_T_MIN = 1.0e-5  # IntersectBvh's default t_min (include/yaoray/accel/bvh.hpp:112)


def sphere_mesh(slices: int = 64, stacks: int = 33):
    """Unit latitude-longitude sphere with fan caps: (positions, triangles)."""
    rings = stacks - 1  # interior latitude rings
    theta = np.pi * (np.arange(1, rings + 1) / stacks)
    phi = 2.0 * np.pi * (np.arange(slices) / slices)
    st, ct = np.sin(theta), np.cos(theta)
    ring = np.stack([np.outer(st, np.cos(phi)), np.repeat(ct[:, None], slices, 1), np.outer(st, np.sin(phi))], -1)
    pos = np.concatenate([[[0.0, 1.0, 0.0]], ring.reshape(-1, 3), [[0.0, -1.0, 0.0]]]).astype(np.float64)
    top, bottom = 0, 1 + rings * slices
    j = np.arange(slices)
    jn = (j + 1) % slices
    tris = [np.stack([np.full(slices, top), 1 + jn, 1 + j], 1)]
    for r in range(rings - 1):
        a = 1 + r * slices + j
        b = 1 + r * slices + jn
        c = 1 + (r + 1) * slices + j
        d = 1 + (r + 1) * slices + jn
        tris.append(np.stack([a, b, d], 1))
        tris.append(np.stack([a, d, c], 1))
    last = 1 + (rings - 1) * slices
    tris.append(np.stack([np.full(slices, bottom), last + j, last + jn], 1))
    return pos, np.concatenate(tris).astype(np.uint32)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def traversal_scene(seed: int = 1, spheres: int = 512, slices: int = 64, stacks: int = 33,
                    box: float = 100.0) -> SceneGeometry:
    """The traversal benchmark geometry (see module docstring)."""
    rng = np.random.default_rng(seed)
    unit_pos, tris = sphere_mesh(slices, stacks)
    nv = unit_pos.shape[0]
    radius = rng.uniform(0.5, 3.0, spheres)
    centre = rng.uniform(0.0, box, (spheres, 3))
    rot = _random_rotations(rng, spheres)
    noise = rng.uniform(-0.05, 0.05, (spheres, nv))
    local = unit_pos[None, :, :] * (radius[:, None, None] * (1.0 + noise[:, :, None]))
    world = np.einsum("sij,svj->svi", rot, local) + centre[:, None, :]
    meshes = [(world[s].astype(np.float32), tris) for s in range(spheres)]
    return SceneGeometry.from_meshes(meshes)


def camera_basis(origin, target, up=(0.0, 1.0, 0.0)):
    o = np.asarray(origin, np.float64)
    f = np.asarray(target, np.float64) - o
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    return o, f, r, u


def coherent_rays(width: int = 2828, height: int = 2828, origin=(50.0, 50.0, 190.0), target=(50.0, 50.0, 50.0),
                  fov_deg: float = 40.0) -> np.ndarray:
    """Pinhole primary rays through pixel centres (GeneratePerspectiveCameraRay
    with a (0.5, 0.5) pixel sample: vertical fov, aspect W/H, y down)."""
    o, f, r, u = camera_basis(origin, target)
    f32 = np.float32
    aspect = f32(width) / f32(height)
    half = f32(np.tan(np.float32(np.radians(fov_deg)) * f32(0.5)))
    xs = (np.arange(width, dtype=f32) + f32(0.5))
    ys = (np.arange(height, dtype=f32) + f32(0.5))
    sx = ((f32(2.0) * xs / f32(width) - f32(1.0)) * aspect * half).astype(f32)
    sy = ((f32(1.0) - f32(2.0) * ys / f32(height)) * half).astype(f32)
    f, r, u = f.astype(f32), r.astype(f32), u.astype(f32)
    d = f[None, None, :] + r[None, None, :] * sx[None, :, None] + u[None, None, :] * sy[:, None, None]
    d = (d / np.sqrt((d * d).sum(-1, keepdims=True))).astype(f32).reshape(-1, 3)
    n = d.shape[0]
    rays = np.empty((n, 8), f32)
    rays[:, 0:3] = o.astype(f32)
    rays[:, 3] = RAY_T_MIN
    rays[:, 4:7] = d
    rays[:, 7] = np.inf
    return rays


def _unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    z = rng.uniform(-1.0, 1.0, n)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    s = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([s * np.cos(phi), s * np.sin(phi), z], 1)


def incoherent_rays(n: int = 2828 * 2828, seed: int = 2, box: float = 100.0) -> np.ndarray:
    """Origins uniform in the box, directions uniform on the sphere."""
    rng = np.random.default_rng(seed)
    rays = np.empty((n, 8), np.float32)
    rays[:, 0:3] = rng.uniform(0.0, box, (n, 3))
    rays[:, 3] = RAY_T_MIN
    rays[:, 4:7] = _unit_vectors(rng, n)
    rays[:, 7] = np.inf
    return rays


def shadow_rays(n: int = 2828 * 2828, seed: int = 3, box: float = 100.0) -> np.ndarray:
    """Any-hit queries: origin uniform in the box towards a uniform random
    point, t_max = distance to it (direction normalised)."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(0.0, box, (n, 3))
    p = rng.uniform(0.0, box, (n, 3))
    d = p - o
    dist = np.linalg.norm(d, axis=1)
    dist = np.maximum(dist, 1e-6)
    rays = np.empty((n, 8), np.float32)
    rays[:, 0:3] = o
    rays[:, 3] = RAY_T_MIN
    rays[:, 4:7] = d / dist[:, None]
    rays[:, 7] = dist
    return rays


def clustered_test_scene() -> SceneGeometry:
    """The reference's clustered 12-triangle test scene
    (tests/accel/bvh_test_scene.hpp:39-53): triangles of half-width 0.25 at
    x offsets {0, .05, .1, .15} + {0, 5, 10}, z = 0, one primitive each."""
    meshes = []
    for off in (0.0, 0.05, 0.10, 0.15, 5.00, 5.05, 5.10, 5.15, 10.00, 10.05, 10.10, 10.15):
        x = np.float32(off)
        p = np.array([[x - np.float32(0.25), -0.25, 0.0], [x + np.float32(0.25), -0.25, 0.0], [x, 0.25, 0.0]],
                     np.float32)
        meshes.append((p, np.array([[0, 1, 2]], np.uint32)))
    return SceneGeometry.from_meshes(meshes)
