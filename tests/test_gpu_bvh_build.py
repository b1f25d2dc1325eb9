"""Device BVH build: the hierarchy built on the GPU is the reference
builder's, byte for byte (nodes, primitive slots, primitives, max depth),
on the traversal set, a Cornell box, spheres, signed zeros, large leaves,
and soups with coincident or nearly coincident centroids (the reference's
median split, whose std::nth_element permutation the host computes)."""
import time

import numpy as np
import pytest

from yaoray_b200 import _lib, accel, cornell, scenes
from yaoray_b200.accel import SceneGeometry

pytestmark = pytest.mark.gpu


def same(a, b):
    assert a.nodes.tobytes() == b.nodes.tobytes()
    assert a.primitive_indices.tobytes() == b.primitive_indices.tobytes()
    assert a.primitives.tobytes() == b.primitives.tobytes()
    assert a.max_depth == b.max_depth


@pytest.mark.parametrize("spheres", [1, 24, 512])
def test_traversal_set_matches_host(spheres):
    geom = scenes.traversal_scene(seed=3, spheres=spheres)
    t0 = time.perf_counter()
    host = accel.build_bvh(geom)
    t1 = time.perf_counter()
    dev, on_device = accel.build_bvh_device(geom)
    t2 = time.perf_counter()
    assert on_device
    same(host, dev)
    print(f"{geom.triangle_count} tris: host {t1 - t0:.3f} s, device {t2 - t1:.3f} s")


def test_cornell_and_large_leaves_match_host():
    geom = cornell.scene(width=8, height=8, spp=1).geometry
    host = accel.build_bvh(geom)
    dev, on_device = accel.build_bvh_device(geom)
    assert on_device
    same(host, dev)
    big = scenes.traversal_scene(seed=9, spheres=8)
    same(accel.build_bvh(big, max_leaf_triangles=100), accel.build_bvh_device(big, max_leaf_triangles=100)[0])


def test_signed_zeros_and_spheres_match_host():
    geom = scenes.traversal_scene(seed=4, spheres=4)
    pos = geom.positions.copy()
    rng = np.random.default_rng(2)
    pick = rng.random(pos.shape) < 0.05
    pos[pick] = 0.0
    pos[pick & (rng.random(pos.shape) < 0.5)] = np.float32(-0.0)
    sp = np.zeros(120, _lib.SPHERE_DTYPE)
    c = np.array([(0.0, -0.0, 1.0), (-0.0, 0.0, -1.0), (3.0, 2.0, 1.0)] * 40, np.float32)
    c[:, 2] += np.repeat(np.arange(40, dtype=np.float32), 3)  # distinct centres, x / y keep their signed zeros
    sp["center"] = c
    sp["radius"] = np.array([0.5, 0.25, 1.0] * 40, np.float32)
    g2 = SceneGeometry(pos, geom.indices, geom.primitives, spheres=sp)
    host = accel.build_bvh(g2)
    dev, on_device = accel.build_bvh_device(g2)
    assert on_device
    same(host, dev)


def test_coincident_centroids_build_on_device():
    """Degenerate ranges (the reference's median split, std::nth_element):
    200 copies of one triangle give ranges above and below the 64-ref small
    subtree size whose centroid extents are all 0. The device build asks the
    host's std::nth_element for the large ones and the host's serial builder
    for the small subtrees, and stays byte-identical to the host builder."""
    geom = scenes.traversal_scene(seed=6, spheres=2)
    pos = geom.positions.copy()
    idx = geom.indices.copy()
    tri = idx[:3]
    idx = np.concatenate([idx, np.tile(tri, 200)])
    prims = geom.primitives.copy()
    prims["index_count"][-1] += 600
    g2 = SceneGeometry(pos, idx, prims)
    host = accel.build_bvh(g2)
    dev, on_device = accel.build_bvh_device(g2)
    assert on_device
    same(host, dev)


def test_nearly_coincident_centroids_build_on_device():
    """Centroids a few 1e-10 apart near the origin: every extent below the
    1e-8 threshold, yet the keys differ, so the median split's permutation
    depends on std::nth_element's own pivoting. 3000 such triangles next to
    an ordinary mesh, byte-identical to the host builder."""
    rng = np.random.default_rng(4)
    base = np.array([[0.0, 0.0, 0.0], [1e-9, 0.0, 0.0], [0.0, 1e-9, 0.0]], np.float32)
    jitter = (rng.random((3000, 1, 3)) * 4e-10).astype(np.float32)
    tris = (base[None] + jitter).reshape(-1, 3).astype(np.float32)
    mesh = scenes.traversal_scene(seed=9, spheres=3)
    g = SceneGeometry.from_meshes([(tris, np.arange(len(tris), dtype=np.uint32).reshape(-1, 3)),
                                   (mesh.positions, mesh.indices.reshape(-1, 3))])
    host = accel.build_bvh(g)
    dev, on_device = accel.build_bvh_device(g)
    assert on_device
    same(host, dev)


def test_two_level_device_matches_host():
    from yaoray_b200 import instanced
    geom = instanced.scene(width=8, height=8, spp=1, mesh_scale=0.1, instances=16, env_width=64).geometry
    host = accel.build_two_level_bvh(geom)
    dev = accel.build_two_level_bvh(geom, device=True)
    assert len(host.blases) == len(dev.blases)
    for (ph, bh, h), (pd, bd, d) in zip(host.blases, dev.blases):
        assert ph == pd and np.array_equal(bh, bd)
        same(h, d)
    assert host.instances.tobytes() == dev.instances.tobytes()
    same(host.tlas, dev.tlas)
