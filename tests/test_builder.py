"""The host builder reproduces the reference's BuildBvh / BuildTwoLevelBvh
layout byte for byte (the GPU kernels consume that layout), including error
strings. Mirrors tests/accel/bvh_builder_tests.cpp and
bvh_parallel_builder_tests.cpp of the reference."""
from pathlib import Path

import numpy as np
import pytest

from yaoray_b200 import YrcError, accel, scenes
from yaoray_b200.accel import SceneGeometry

GOLDEN = Path(__file__).resolve().parent / "golden"


def golden_geometry(name):
    f = dict(np.load(GOLDEN / f"{name}.npz"))
    return f, SceneGeometry(f["positions"], f["indices"], f["primitives"], f["spheres"], f["instances"])


@pytest.mark.parametrize("name", ["trace_clustered", "trace_spheres"])
def test_flat_build_matches_reference_golden(name):
    f, g = golden_geometry(name)
    b = accel.build_bvh(g)
    assert b.nodes.tobytes() == f["bvh_nodes"].tobytes()
    assert b.primitive_indices.tobytes() == f["bvh_primitive_indices"].tobytes()
    assert b.primitives.tobytes() == f["bvh_primitives"].tobytes()
    assert b.max_depth == int(f["bvh_max_depth"])


def test_single_leaf_and_leaf_size():
    # bvh_builder_tests.cpp: max_leaf_triangles=4 -> 3 triangles share 1 leaf.
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    g = SceneGeometry.from_meshes([(p + [i, 0, 0], [[0, 1, 2]]) for i in range(3)])
    b = accel.build_bvh(g)
    assert len(b.nodes) == 1 and b.nodes[0]["primitive_count"] == 3
    assert b.max_depth == 1 and b.total_triangles == 3


def test_sah_has_fewer_nodes_than_median_on_clusters():
    g = scenes.clustered_test_scene()
    sah = accel.build_bvh(g, "sah")
    med = accel.build_bvh(g, "median")
    assert len(sah.nodes) < len(med.nodes)


def test_degenerate_centroids_still_build():
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    g = SceneGeometry.from_meshes([(p, [[0, 1, 2]]) for _ in range(9)])
    b = accel.build_bvh(g)
    assert b.total_triangles == 9
    assert (b.nodes["primitive_count"] > 0).sum() >= 1
    assert sorted(b.primitive_indices.tolist()) == list(range(9))


def test_parallel_equals_serial_bytes():
    g = scenes.traversal_scene(seed=3, spheres=40, slices=32, stacks=17)
    serial = accel.build_bvh(g, thread_count=1)
    for threads in (2, 3, 8):
        par = accel.build_bvh(g, thread_count=threads, parallel_min_subtree_size=64)
        assert par.nodes.tobytes() == serial.nodes.tobytes()
        assert par.primitive_indices.tobytes() == serial.primitive_indices.tobytes()
        assert par.max_depth == serial.max_depth


def test_empty_geometry_builds_empty_bvh():
    g = SceneGeometry.from_meshes([])
    b = accel.build_bvh(g)
    assert len(b.nodes) == 0 and len(b.primitives) == 0


@pytest.mark.parametrize("mutate,message", [
    (lambda g: g.primitives.__setitem__("index_count", 4), "non-triangular index count"),
    (lambda g: g.primitives.__setitem__("first_index", 99), "invalid index range"),
    (lambda g: g.indices.__setitem__(1, 77), "invalid vertex index"),
    (lambda g: g.positions.__setitem__((0, 0), np.nan), "non-finite triangle data"),
])
def test_build_errors_use_reference_strings(mutate, message):
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1, 1, 0]], np.float32)
    g = SceneGeometry.from_meshes([(p, [[0, 1, 2], [1, 3, 2]])])
    mutate(g)
    with pytest.raises(YrcError, match=message):
        accel.build_bvh(g)


def test_invalid_sphere_and_options_errors():
    g = SceneGeometry.from_meshes([], spheres=[[0, 0, 0, -1.0]])
    with pytest.raises(YrcError, match="invalid sphere data"):
        accel.build_bvh(g)
    g = SceneGeometry.from_meshes([], spheres=[[0, 0, 0, 1.0]])
    with pytest.raises(YrcError, match="max_leaf_triangles must be at least 1"):
        accel.build_bvh(g, max_leaf_triangles=0)


def test_two_level_identity_and_reuse():
    # two_level_bvh_tests.cpp: identity instances are synthesised; one BLAS
    # serves several instances.
    p = np.array([[-0.25, -0.25, 0], [0.25, -0.25, 0], [0, 0.25, 0]], np.float32)
    g = SceneGeometry.from_meshes([(p, [[0, 1, 2]])])
    tl = accel.build_two_level_bvh(g)
    assert len(tl.blases) == 1 and tl.instances.size == 1
    m = np.eye(4, dtype=np.float32)
    inst = []
    for dx in (-1.0, 1.0):
        mm = m.copy()
        mm[:3, 3] = (dx, 0, 0)
        inst.append((0, mm.T.reshape(16)))
    g2 = SceneGeometry.from_meshes([(p, [[0, 1, 2]])], instances=inst)
    tl2 = accel.build_two_level_bvh(g2)
    assert len(tl2.blases) == 1 and tl2.instances.size == 2


def test_two_level_rejects_singular_transform():
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    g = SceneGeometry.from_meshes([(p, [[0, 1, 2]])], instances=[(0, np.zeros(16, np.float32))])
    with pytest.raises(YrcError, match="singular or non-finite"):
        accel.build_two_level_bvh(g)
    g = SceneGeometry.from_meshes([(p, [[0, 1, 2]])], instances=[(3, np.eye(4, dtype=np.float32).reshape(16))])
    with pytest.raises(YrcError, match="invalid mesh primitive"):
        accel.build_two_level_bvh(g)


def test_flat_build_matches_live_reference(ref):
    for seed in (1, 2):
        g = scenes.traversal_scene(seed=seed, spheres=64, slices=24, stacks=13)
        for split in ("sah", "median"):
            ours = accel.build_bvh(g, split)
            nodes, pi, prims, md = ref.RefScene(g, split_method=split).flat_bvh()
            assert ours.nodes.tobytes() == nodes.tobytes()
            assert ours.primitive_indices.tobytes() == pi.tobytes()
            assert ours.primitives.tobytes() == prims.tobytes()
            assert ours.max_depth == md


def test_median_splits_match_live_reference(ref):
    """Nearly coincident centroids (extents below the reference's 1e-8, keys
    still distinct): the median split's std::nth_element permutation, which
    the host builder and the device builder's host step both take from the
    standard library, gives the reference's bytes."""
    rng = np.random.default_rng(4)
    base = np.array([[0.0, 0.0, 0.0], [1e-9, 0.0, 0.0], [0.0, 1e-9, 0.0]], np.float32)
    tris = (base[None] + (rng.random((3000, 1, 3)) * 4e-10).astype(np.float32)).reshape(-1, 3).astype(np.float32)
    mesh = scenes.traversal_scene(seed=9, spheres=3)
    g = SceneGeometry.from_meshes([(tris, np.arange(len(tris), dtype=np.uint32).reshape(-1, 3)),
                                   (mesh.positions, mesh.indices.reshape(-1, 3))])
    b = accel.build_bvh(g)
    nodes, pi, prims, depth = ref.RefScene(g).flat_bvh()
    assert b.nodes.tobytes() == nodes.tobytes() and b.primitive_indices.tobytes() == pi.tobytes()
    assert b.primitives.tobytes() == prims.tobytes() and b.max_depth == depth


def test_two_level_build_matches_live_reference(ref):
    f, g = golden_geometry("trace_two_level")
    ours = accel.build_two_level_bvh(g)
    theirs = ref.RefScene(g).two_level_bvh()
    assert ours.tlas.nodes.tobytes() == theirs["tlas_nodes"].tobytes()
    assert ours.tlas.primitive_indices.tobytes() == theirs["tlas_primitive_indices"].tobytes()
    assert ours.tlas.max_depth == theirs["tlas_max_depth"]
    for (mp, bounds, b), (rmp, rb, rn, rpi, rpr, rmd) in zip(ours.blases, theirs["blases"]):
        assert mp == rmp and b.nodes.tobytes() == rn.tobytes() and b.primitives.tobytes() == rpr.tobytes()
        assert bounds.tobytes() == rb.tobytes()
    for key, ours_key in (("world_to_object", "world_to_object"), ("object_to_world", "object_to_world")):
        assert ours.instances[ours_key].reshape(-1, 16).tobytes() == theirs[key].tobytes()
    assert np.concatenate([ours.instances["world_bounds_min"], ours.instances["world_bounds_max"]], 1).tobytes() == \
        theirs["world_bounds"].tobytes()
