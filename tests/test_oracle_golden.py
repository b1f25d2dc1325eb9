"""Pins the oracle restatement (oracle/yr_oracle.c) to golden vectors produced
by the reference implementation (tests/golden/make_golden.py), and — where the
compiled reference is present — directly against it on fresh seeded inputs."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from yaoray_b200 import accel, scenes
from yaoray_b200.accel import RenderBvh, SceneGeometry

GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def geometry(f) -> SceneGeometry:
    return SceneGeometry(f["positions"], f["indices"], f["primitives"], f["spheres"], f["instances"])


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def assert_trace_equal(hits, st, f):
    assert np.array_equal(hits["hit"].astype(bool), f["out_hit"].astype(bool))
    assert np.array_equal(hits["triangle_index"], f["out_triangle_index"])
    assert np.array_equal(hits["sphere"], f["out_sphere"])
    assert np.array_equal(hits["mesh_primitive"], f["out_mesh_primitive"])
    assert np.array_equal(hits["instance"], f["out_instance"])
    assert np.array_equal(bits(hits["t"]), bits(f["out_t"]))
    tri = f["out_triangle_index"] >= 0
    assert np.array_equal(bits(hits["u"][tri]), bits(f["out_u"][tri]))
    assert np.array_equal(bits(hits["v"][tri]), bits(f["out_v"][tri]))
    assert np.array_equal(st[0], f["out_node_tests"])
    assert np.array_equal(st[1], f["out_triangle_tests"])
    assert np.array_equal(st[2], f["out_sphere_tests"])


@pytest.mark.parametrize("name", ["trace_clustered", "trace_spheres"])
def test_flat_trace_matches_reference_golden(name):
    f = load(name)
    bvh = RenderBvh(f["bvh_nodes"], f["bvh_primitive_indices"], f["bvh_primitives"], int(f["bvh_max_depth"]))
    hits, st = oracle.OracleScene(geometry(f), bvh).trace(f["rays"], threads=2)
    assert_trace_equal(hits, st, f)


def test_clustered_reference_pins():
    # bvh_traversal_tests.cpp:91-138: the cluster at x=5 is hit by the ray
    # from (5,0,1); the ray at x=50 misses.
    f = load("trace_clustered")
    assert f["out_hit"][0] and f["out_triangle_index"][0] == 0
    assert abs(f["out_t"][0] - 1.0) < 1e-6
    assert f["out_hit"][1] and f["out_triangle_index"][1] == 4
    assert not f["out_hit"][2]


def test_spheres_golden_covers_edge_cases():
    f = load("trace_spheres")
    assert f["out_hit"].mean() > 0.1
    assert (f["out_sphere"] >= 0).sum() > 10, "analytic sphere hits are exercised"
    r = f["rays"]
    assert (r[:, 7] == 0).any() and np.isinf(r[:, 7]).any()
    assert (np.signbit(r[:, 4:7]) & (r[:, 4:7] == 0)).any(), "negative-zero directions are exercised"


def test_two_level_trace_matches_reference_golden():
    f = load("trace_two_level")
    g = geometry(f)
    tl = accel.build_two_level_bvh(g)
    assert tl.tlas.nodes.tobytes() == f["tlas_nodes"].tobytes()
    assert np.array_equal(bits(tl.instances["world_to_object"].reshape(-1, 16)), bits(f["world_to_object"]))
    hits, st = oracle.OracleScene(g, tl).trace(f["rays"], threads=2)
    assert_trace_equal(hits, st, f)
    assert (f["out_instance"] >= 0).sum() > 50


def test_probe_matches_reference_golden():
    f = load("probe_layers")
    g = geometry(f)
    bvh = accel.build_bvh(g)
    hits, counts, ex = oracle.OracleScene(g, bvh).probe(f["rays"], f["targets"])
    assert np.array_equal(counts, f["out_count"])
    assert np.array_equal(ex, f["out_exhausted"])
    for i in np.nonzero(counts)[0]:
        c = counts[i]
        assert np.array_equal(bits(hits["t"][i, :c]), bits(f["out_t"][i, :c]))
        assert np.array_equal(hits["triangle_index"][i, :c], f["out_triangle_index"][i, :c])
    assert counts.max() >= 2


@pytest.mark.parametrize("kind", [0, 1, 2, 3])
def test_sampler_matches_reference_golden(kind):
    f = load("sampler")
    for seed in (0, 0x5EED1234):
        for spp in (1, 64):
            for d2 in (False, True):
                key = f"k{kind}_s{seed}_p{spp}_{'2d' if d2 else '1d'}"
                got = oracle.oracle_sampler(kind, seed, spp, f["queries"], d2)
                assert np.array_equal(bits(got), bits(f[key])), key


def test_rng_and_pixel_seed_match_reference_golden():
    f = load("sampler")
    for s, draws in zip(f["rng_seeds"], f["rng_draws"]):
        assert np.array_equal(bits(oracle.oracle_rng(int(s), 16)), bits(draws))
    for (x, y, smp), v in zip(f["seed_pixel_queries"], f["seed_pixel_values"]):
        assert oracle.oracle_seed_for_pixel_sample(0x1234, int(x), int(y), int(smp)) == int(v)


def test_camera_matches_reference_golden():
    f = load("camera_film")
    got = oracle.oracle_camera_rays(f["camera"], 256, 256, f["pixels"], f["samples"])
    assert np.array_equal(bits(got), bits(f["rays"]))


def test_film_matches_reference_golden():
    f = load("camera_film")
    px, bad = oracle.oracle_film(int(f["film_w"]), int(f["film_h"]), f["film_samples"])
    assert bad == int(f["film_bad"])
    assert px.view(np.uint8).tobytes() == f["film_pixels"].tobytes()


def same_values(a, b):
    """Bit-equal, except that any NaN matches any NaN (x86-64 and CUDA
    produce NaNs with different payloads)."""
    a = np.ascontiguousarray(a, np.float32)
    b = np.ascontiguousarray(b, np.float32)
    na, nb = np.isnan(a), np.isnan(b)
    return np.array_equal(na, nb) and np.array_equal(bits(np.where(na, 0, a)), bits(np.where(nb, 0, b)))


def test_texture_matches_reference_golden():
    f = load("texture")
    for si in range(len(f["shapes"])):
        tx = f[f"t{si}_texels"]
        for wi, (ws, wt) in enumerate(f["wraps"]):
            uv, fp = f[f"t{si}_w{wi}_uv"], f[f"t{si}_w{wi}_fp"]
            for filt in range(4):
                got = oracle.oracle_texture_sample(tx, filt, int(ws), int(wt), uv, fp)
                assert same_values(got, f[f"t{si}_w{wi}_f{filt}"]), (si, wi, filt)
            mips = oracle.oracle_texture_mip_chain(tx, int(ws), int(wt))
            expect = [f[k] for k in sorted((k for k in f if k.startswith(f"t{si}_w{wi}_mip")),
                                           key=lambda k: int(k.split("mip")[1]))]
            assert len(mips) == len(expect)
            for a, b in zip(mips, expect):
                assert np.array_equal(bits(a), bits(b))


# ---------------------------------------------------------- live reference

def test_oracle_matches_live_reference_on_traversal_set(ref):
    g = scenes.traversal_scene(seed=31, spheres=48, slices=32, stacks=17)
    bvh = accel.build_bvh(g)
    rays = np.concatenate([scenes.incoherent_rays(20000, seed=32), scenes.coherent_rays(96, 96),
                           scenes.shadow_rays(10000, seed=33)])
    r = ref.RefScene(g).trace(rays)
    hits, st = oracle.OracleScene(g, bvh).trace(rays)
    assert np.array_equal(hits["triangle_index"], r["triangle_index"])
    assert np.array_equal(bits(hits["t"]), bits(r["t"]))
    assert np.array_equal(st[0], r["node_tests"]) and np.array_equal(st[1], r["triangle_tests"])


def test_oracle_sampler_matches_live_reference_random(ref):
    rng = np.random.default_rng(7)
    q = np.stack([rng.integers(0, 2000, 5000), rng.integers(0, 2000, 5000), rng.integers(0, 4096, 5000),
                  rng.integers(0, 16, 5000), rng.integers(0, 16, 5000), rng.integers(0, 4, 5000)], 1)
    for kind in (2, 3):
        for spp in (16, 1024):
            for d2 in (False, True):
                a = oracle.oracle_sampler(kind, 99, spp, q, d2)
                b = ref.ref_sampler(kind, 99, spp, q, d2)
                assert np.array_equal(bits(a), bits(b))


def test_oracle_texture_matches_live_reference_random(ref):
    rng = np.random.default_rng(12)
    for h, w in [(3, 7), (64, 48), (1, 129)]:
        tx = rng.random((h, w, 4), dtype=np.float32)
        uv = rng.uniform(-4, 4, (4000, 2)).astype(np.float32)
        fp = (rng.standard_normal((4000, 4)) * np.exp(rng.uniform(-9, 1, (4000, 1)))).astype(np.float32)
        for ws, wt in [(0, 1), (2, 0), (1, 2)]:
            for filt in range(4):
                a = oracle.oracle_texture_sample(tx, filt, ws, wt, uv, fp)
                b = ref.ref_texture_sample(tx, filt, ws, wt, uv, fp)
                assert same_values(a, b), (h, w, ws, wt, filt)
