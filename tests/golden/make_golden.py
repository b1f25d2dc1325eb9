"""Generates tests/golden/*.npz from the REFERENCE implementation itself.

The reference ships no golden vectors (its tests are property pins), so the
fixtures are outputs of the unmodified reference code, compiled from its
sources by oracle/Makefile into oracle/_ref/libyaoray_ref.so and called
through oracle/ref_shim.cpp: IntersectAcceleration / IntersectTwoLevelBvh /
IntersectAccelerationProbe, BuildBvh / BuildTwoLevelBvh, Sampler, Rng,
GeneratePerspectiveCameraRay, Film::AddSample, SampleTexture4 and
BuildTextureMipChain. Inputs are small seeded
cases; each file stores inputs and expected outputs so the CPU tests can pin
the oracle restatement without the reference present.

Run: python tests/golden/make_golden.py [texture|measured]   (needs oracle/_ref
built; `texture` / `measured` write only that fixture)
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

import oracle  # noqa: E402
from yaoray_b200 import scenes  # noqa: E402
from yaoray_b200.accel import SceneGeometry  # noqa: E402


def _geometry_arrays(g: SceneGeometry) -> dict:
    return {"positions": g.positions, "indices": g.indices, "primitives": g.primitives, "spheres": g.spheres,
            "instances": g.instances}


def edge_rays(rng: np.random.Generator, n: int, lo: float, hi: float) -> np.ndarray:
    """Rays exercising the slab test's special cases: zero and negative-zero
    direction components (1/d = +-inf), rays starting on the box planes,
    narrow [t_min, t_max] windows and t_max = 0."""
    r = np.zeros((n, 8), np.float32)
    r[:, 0:3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    axis = rng.integers(0, 3, n)
    kind = rng.integers(0, 4, n)
    d[kind == 0, :] = 0.0
    d[kind == 0, axis[kind == 0]] = rng.choice([-1.0, 1.0], (kind == 0).sum())
    d[kind == 1, axis[kind == 1]] = 0.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r[:, 4:7] = d
    neg0 = kind == 2
    r[neg0, 4 + axis[neg0]] = np.float32(-0.0)
    r[:, 3] = 1.0e-5
    r[:, 7] = np.inf
    win = rng.random(n) < 0.25
    r[win, 3] = rng.uniform(0.0, 20.0, win.sum())
    r[win, 7] = r[win, 3] + rng.uniform(0.0, 30.0, win.sum())
    zero = rng.random(n) < 0.05
    r[zero, 7] = 0.0
    return r


def trace_fixture(name: str, g: SceneGeometry, rays: np.ndarray) -> None:
    ref = oracle.RefScene(g)
    assert ref.errors == 0, ref.error
    out = ref.trace(rays, threads=1)
    arrays = {"rays": rays, **_geometry_arrays(g), **{f"out_{k}": v for k, v in out.items()}}
    if ref.two_level:
        tl = ref.two_level_bvh()
        arrays["tlas_nodes"] = tl["tlas_nodes"]
        arrays["world_to_object"] = tl["world_to_object"]
    else:
        nodes, pi, prims, md = ref.flat_bvh()
        arrays.update({"bvh_nodes": nodes, "bvh_primitive_indices": pi, "bvh_primitives": prims,
                       "bvh_max_depth": np.int32(md)})
    np.savez_compressed(HERE / f"{name}.npz", **arrays)


def main() -> None:
    rng = np.random.default_rng(20261203)

    # 1. The reference's clustered 12-triangle scene and its test rays
    #    (tests/accel/bvh_traversal_tests.cpp:91-138) plus random probes.
    g = scenes.clustered_test_scene()
    fixed = np.array([[0, 0, 1, 1e-5, 0, 0, -1, np.inf], [5, 0, 1, 1e-5, 0, 0, -1, np.inf],
                      [50, 0, 1, 1e-5, 0, 0, -1, np.inf]], np.float32)
    rnd = np.zeros((400, 8), np.float32)
    rnd[:, 0] = rng.uniform(-1, 11, 400)
    rnd[:, 1] = rng.uniform(-0.5, 0.5, 400)
    rnd[:, 2] = rng.uniform(0.5, 2.0, 400)
    rnd[:, 3] = 1e-5
    d = np.stack([rng.normal(0, 0.1, 400), rng.normal(0, 0.1, 400), -np.ones(400)], 1)
    rnd[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rnd[:, 7] = np.inf
    trace_fixture("trace_clustered", g, np.concatenate([fixed, rnd]))

    # 2. Noisy spheres (16 x 256 triangles) + two analytic spheres.
    g = scenes.traversal_scene(seed=11, spheres=16, slices=16, stacks=9, box=20.0)
    sph = np.zeros(2, g.spheres.dtype)
    sph["center"] = [[5.0, 5.0, 5.0], [14.0, 12.0, 9.0]]
    sph["radius"] = [1.5, 2.5]
    sph["area_light_index"] = -1
    g = SceneGeometry(g.positions, g.indices, g.primitives, sph)
    rays = np.concatenate([scenes.incoherent_rays(1500, seed=12, box=20.0),
                           scenes.coherent_rays(32, 24, origin=(10, 10, 45), target=(10, 10, 10)),
                           scenes.shadow_rays(800, seed=13, box=20.0),
                           edge_rays(rng, 700, 0.0, 20.0)])
    trace_fixture("trace_spheres", g, rays)

    # 3. Two-level: 2 meshes, 7 affine instances (rotation, non-uniform
    #    scale, translation) and one analytic sphere in the TLAS.
    base = scenes.traversal_scene(seed=21, spheres=2, slices=12, stacks=7, box=4.0)
    inst = np.zeros(7, g.instances.dtype)
    for k in range(7):
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                      [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                      [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
        M = np.eye(4)
        M[:3, :3] = R @ np.diag(rng.uniform(0.5, 2.0, 3))
        M[:3, 3] = rng.uniform(0.0, 20.0, 3)
        inst[k]["primitive"] = k % 2
        inst[k]["object_to_world"] = M.T.reshape(16).astype(np.float32)  # column-major
    sph = np.zeros(1, g.spheres.dtype)
    sph["center"] = [[10.0, 10.0, 10.0]]
    sph["radius"] = [1.0]
    sph["area_light_index"] = -1
    g2 = SceneGeometry(base.positions, base.indices, base.primitives, sph, inst)
    rays = np.concatenate([scenes.incoherent_rays(1500, seed=22, box=20.0), scenes.shadow_rays(500, seed=23, box=20.0),
                           edge_rays(rng, 300, 0.0, 20.0)])
    trace_fixture("trace_two_level", g2, rays)

    # 4. Probe: stacked quads (the reference's probe test shape) + spheres.
    quads = []
    for z in (0.0, 0.5, 2.0):
        p = np.array([[-1, -1, z], [1, -1, z], [1, 1, z], [-1, 1, z]], np.float32)
        quads.append((p, np.array([[0, 1, 2], [0, 2, 3]], np.uint32)))
    # primitive 0 and 2 are layered targets, primitive 1 sits between them
    layered = np.concatenate([quads[0][0], quads[2][0]])
    meshes = [(layered, np.array([[0, 1, 2], [0, 2, 3], [4, 5, 6], [4, 6, 7]], np.uint32)), quads[1]]
    gp = SceneGeometry.from_meshes(meshes, spheres=[[0.0, 0.0, 4.0, 0.5]])
    n = 256
    pr = np.zeros((n, 8), np.float32)
    pr[:, 0] = rng.uniform(-1.2, 1.2, n)
    pr[:, 1] = rng.uniform(-1.2, 1.2, n)
    pr[:, 2] = -1.0
    pr[:, 3] = 1e-5
    pr[:, 6] = 1.0
    pr[:, 7] = rng.choice([1.0, 3.0, 10.0], n)
    targets = np.zeros((n, 4), np.int32)
    targets[:, 0] = rng.choice([-1, 0, 1], n)
    targets[:, 1] = -1
    targets[:, 2] = np.where(targets[:, 0] < 0, 0, -1)
    ref = oracle.RefScene(gp)
    out = ref.probe(pr, targets)
    np.savez_compressed(HERE / "probe_layers.npz", rays=pr, targets=targets, **_geometry_arrays(gp),
                        **{f"out_{k}": v for k, v in out.items()})

    # 5. Sampler: all four kinds, 1-D and 2-D, semantic dimensions x bounces.
    dims = np.array([0, 2, 3, 5, 7, 8, 9, 10, 12, 14])
    q = np.stack([rng.integers(0, 300, 3000), rng.integers(0, 300, 3000), rng.integers(0, 128, 3000),
                  rng.integers(0, 12, 3000), rng.choice(dims, 3000), rng.integers(0, 3, 3000)], 1).astype(np.int32)
    fx = {"queries": q}
    for kind in (0, 1, 2, 3):
        for seed in (0, 0x5EED1234):
            for spp in (1, 64):
                fx[f"k{kind}_s{seed}_p{spp}_1d"] = oracle.ref_sampler(kind, seed, spp, q, False)
                fx[f"k{kind}_s{seed}_p{spp}_2d"] = oracle.ref_sampler(kind, seed, spp, q, True)
    seeds = rng.integers(0, 2**63, 64, dtype=np.uint64)
    fx["rng_seeds"] = seeds
    fx["rng_draws"] = np.stack([oracle.ref_rng(int(s), 16) for s in seeds])
    pix = np.stack([rng.integers(-5, 4000, 64), rng.integers(-5, 4000, 64), rng.integers(0, 5000, 64)], 1)
    fx["seed_pixel_queries"] = pix
    fx["seed_pixel_values"] = np.array([oracle.ref_seed_for_pixel_sample(0x1234, int(a), int(b), int(c))
                                        for a, b, c in pix], np.uint64)
    np.savez_compressed(HERE / "sampler.npz", **fx)

    # 6. Camera rays and film accumulation.
    cam = np.array([2.78, 2.73, -8.0, 0, 0, 1, -1, 0, 0, 0, 1, 0, np.radians(40.0)], np.float32)
    px = np.stack([rng.integers(0, 256, 2000), rng.integers(0, 256, 2000)], 1).astype(np.int32)
    sm = rng.random((2000, 2)).astype(np.float32)
    cam_rays = oracle.ref_camera_rays(cam, 256, 256, px, sm)
    w, h = 16, 12
    s = np.zeros((5000, 13), np.float32)
    s[:, 0] = rng.integers(0, w, 5000)
    s[:, 1] = rng.integers(0, h, 5000)
    s[:, 2:5] = rng.exponential(1.0, (5000, 3))
    s[:, 5:8] = rng.random((5000, 3))
    s[:, 8:11] = rng.normal(size=(5000, 3))
    s[:, 11] = rng.uniform(-1, 10, 5000)
    s[:, 12] = rng.random(5000) < 0.7
    bad = rng.random(5000) < 0.02
    s[bad, 2 + rng.integers(0, 3, bad.sum())] = np.float32(np.nan)
    s[rng.random(5000) < 0.01, 3] = np.float32(np.inf)
    s[rng.random(5000) < 0.02, 8] = np.float32(np.nan)
    film, nbad = oracle.ref_film(w, h, s)
    np.savez_compressed(HERE / "camera_film.npz", camera=cam, pixels=px, samples=sm, rays=cam_rays, film_samples=s,
                        film_w=w, film_h=h, film_pixels=film.view(np.uint8), film_bad=np.int64(nbad))
    texture_fixture()
    measured_fixture()
    print("golden fixtures written to", HERE)


def texture_fixture() -> None:
    """7. Texture lookups (SampleTexture4 after BuildTextureSamplingCaches)
    and mip chains (BuildTextureMipChain): odd and degenerate sizes, every
    wrap mode, every filter, lookups with and without footprints, uvs on
    texel edges, far outside [0, 1] and non-finite."""
    rng = np.random.default_rng(0x7E57)
    shapes = [(1, 1), (1, 37), (37, 1), (2, 2), (4, 4), (5, 3), (23, 37), (32, 32)]
    wraps = [(0, 0), (1, 1), (2, 2), (0, 2), (2, 1)]
    fx = {"shapes": np.array(shapes, np.int32), "wraps": np.array(wraps, np.int32)}
    n = 160
    for si, (h, w) in enumerate(shapes):
        tx = rng.random((h, w, 4), dtype=np.float32)
        tx[..., 3] = rng.choice(np.array([0.0, 0.3, 0.7, 1.0], np.float32), (h, w))
        fx[f"t{si}_texels"] = tx
        for wi, (ws, wt) in enumerate(wraps):
            uv = rng.uniform(-2.5, 3.5, (n, 2)).astype(np.float32)
            uv[:16] = rng.integers(-3 * w, 4 * w, (16, 2)) / np.array([w, h], np.float32)
            uv[16:20] = np.array([[0, 0], [1, 1], [0.5, 0.5], [1e3, -1e3]], np.float32)
            uv[20:22] = np.array([[np.nan, 0.25], [np.inf, 0.5]], np.float32)
            fp = (rng.standard_normal((n, 4)) * np.exp(rng.uniform(-10.0, 2.0, (n, 1)))).astype(np.float32)
            fp[:40] = 0.0
            fp[40:50, 1:3] = 0.0  # axis-aligned footprints
            fx[f"t{si}_w{wi}_uv"] = uv
            fx[f"t{si}_w{wi}_fp"] = fp
            for f in range(4):
                fx[f"t{si}_w{wi}_f{f}"] = oracle.ref_texture_sample(tx, f, ws, wt, uv, fp)
            for li, lv in enumerate(oracle.ref_texture_mip_chain(tx, ws, wt)):
                fx[f"t{si}_w{wi}_mip{li}"] = lv
    np.savez_compressed(HERE / "texture.npz", **fx)


def measured_fixture() -> None:
    """8. Measured BRDF: EvaluateMeasured / PdfMeasured / SampleMeasured of
    the seeded synthetic RGL-layout BRDF (yaoray_b200.measured.synthetic_brdf
    seed 5, rebuilt from its seed by the tests) on seeded directions."""
    from yaoray_b200 import measured as M

    rng = np.random.default_rng(0xB8DF)
    brdf = M.synthetic_brdf(5)
    n = 4000
    nrm = rng.normal(size=(n, 3))
    nrm = (nrm / np.linalg.norm(nrm, axis=1, keepdims=True)).astype(np.float32)
    wo = nrm * rng.uniform(0.05, 1.0, (n, 1)) + rng.normal(size=(n, 3)) * 0.6
    wo = (wo / np.linalg.norm(wo, axis=1, keepdims=True)).astype(np.float32)
    wi = nrm * rng.uniform(-0.2, 1.0, (n, 1)) + rng.normal(size=(n, 3)) * 0.6
    wi = (wi / np.linalg.norm(wi, axis=1, keepdims=True)).astype(np.float32)
    u = rng.random((n, 2)).astype(np.float32)
    f, pdf = oracle.ref_measured_eval(brdf, wo, wi, nrm)
    smp = oracle.ref_measured_sample(brdf, wo, nrm, u)
    np.savez_compressed(HERE / "measured.npz", seed=np.int64(5), wo=wo, wi=wi, n=nrm, u=u, f=f, pdf=pdf, sample=smp)


if __name__ == "__main__":
    if sys.argv[1:] == ["texture"]:
        texture_fixture()
    elif sys.argv[1:] == ["measured"]:
        measured_fixture()
    else:
        main()
