"""GPU traversal parity: the CUDA kernels (through the C ABI) against the
oracle — bit-exact hit IDs, t and barycentrics, node/triangle test counts,
any-hit occlusion — on golden fixtures, the full-size traversal set and edge
cases. Analytic-sphere UVs go through CUDA atan2f/acosf, whose results differ
from the host libm's in the last bits (up to ~1.3e-6 absolute has been
seen), so they are compared with an absolute tolerance of 4e-6; every other
output is compared bit for bit."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from yaoray_b200 import accel, scenes
from yaoray_b200.accel import RenderBvh, SceneGeometry

pytestmark = pytest.mark.gpu
GOLDEN = Path(__file__).resolve().parent / "golden"


def load(name):
    return dict(np.load(GOLDEN / f"{name}.npz"))


def geometry(f):
    return SceneGeometry(f["positions"], f["indices"], f["primitives"], f["spheres"], f["instances"])


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def expected_ids(h):
    tri = np.asarray(h["triangle_index"])
    sph = np.asarray(h["sphere"])
    hit = np.asarray(h["hit"]).astype(bool)
    return np.where(hit, np.where(tri >= 0, tri, -2 - sph), -1).astype(np.int32)


def check_closest(hits, inst, exp, exp_inst=None):
    hits = hits.cpu().numpy() if not isinstance(hits, np.ndarray) else hits
    ids = accel.hit_ids(hits)
    want = expected_ids(exp)
    mism = np.nonzero(ids != want)[0]
    assert mism.size == 0, f"{mism.size} id mismatches, first {mism[:5]}: got {ids[mism[:5]]} want {want[mism[:5]]}"
    assert np.array_equal(bits(hits[:, 0]), bits(exp["t"])), "t not bit-identical"
    tri = want >= 0
    assert np.array_equal(bits(hits[tri, 2]), bits(np.asarray(exp["u"])[tri])), "u not bit-identical"
    assert np.array_equal(bits(hits[tri, 3]), bits(np.asarray(exp["v"])[tri])), "v not bit-identical"
    sph = want <= -2
    if sph.any():
        assert np.abs(hits[sph, 2] - np.asarray(exp["u"])[sph]).max() <= 4e-6
        assert np.abs(hits[sph, 3] - np.asarray(exp["v"])[sph]).max() <= 4e-6
    if exp_inst is not None:
        got_inst = inst.cpu().numpy()
        assert np.array_equal(got_inst, np.where(want != -1, exp_inst, -1))


def golden_accel(f, name):
    g = geometry(f)
    if "bvh_nodes" in f:
        b = RenderBvh(f["bvh_nodes"], f["bvh_primitive_indices"], f["bvh_primitives"], int(f["bvh_max_depth"]))
    else:
        b = accel.build_two_level_bvh(g)
    return g, b


@pytest.mark.parametrize("name", ["trace_clustered", "trace_spheres", "trace_two_level"])
def test_golden_closest_any_and_stats(cuda, name):
    import torch

    f = load(name)
    g, b = golden_accel(f, name)
    dev = accel.DeviceAccelerator(g, b)
    rays = torch.from_numpy(f["rays"]).to(cuda)
    inst = torch.empty(rays.shape[0], dtype=torch.int32, device=cuda)
    hits = dev.intersect(rays, instances=inst)
    occ = dev.intersect(rays, any_hit=True)
    st = dev.trace_stats(rays).cpu().numpy()
    st_any = dev.trace_stats(rays, any_hit=True).cpu().numpy()
    dev.check()
    exp = {k[4:]: v for k, v in f.items() if k.startswith("out_")}
    check_closest(hits, inst, exp, exp["instance"])
    assert np.array_equal(occ.cpu().numpy().astype(bool), exp["hit"].astype(bool))
    assert np.array_equal(st[0], exp["node_tests"])
    assert np.array_equal(st[1], exp["triangle_tests"])
    assert np.array_equal(st[2], exp["sphere_tests"])
    # any-hit stops at the first accepted primitive: never more work
    assert (st_any[0] <= st[0]).all() and (st_any[1] <= st[1]).all()


@pytest.mark.parametrize("name", ["trace_spheres", "trace_two_level"])
def test_golden_host_path_matches(cuda, name):
    f = load(name)
    g, b = golden_accel(f, name)
    dev = accel.DeviceAccelerator(g, b)
    rays = np.ascontiguousarray(f["rays"])
    inst = np.empty(rays.shape[0], np.int32)
    hits, stats = dev.intersect_host(rays, with_stats=True, instances_out=inst)
    exp = {k[4:]: v for k, v in f.items() if k.startswith("out_")}
    check_closest(hits, None, exp)
    assert stats["node_tests"] == int(exp["node_tests"].sum())
    assert stats["triangle_tests"] == int(exp["triangle_tests"].sum())
    occ = dev.intersect_host(rays, any_hit=True)
    assert np.array_equal(occ.astype(bool), exp["hit"].astype(bool))


@pytest.mark.parametrize("name", ["trace_spheres", "trace_two_level"])
def test_host_path_autotune_keeps_the_reference_hits(cuda, name):
    """The host path's own launch shape (tuned on the host pipeline) changes
    no hit: after autotune_host, and with every shape set explicitly, the
    host path returns the reference's hits and occlusion."""
    import torch

    f = load(name)
    g, b = golden_accel(f, name)
    dev = accel.DeviceAccelerator(g, b)
    rays = torch.from_numpy(np.ascontiguousarray(f["rays"])).pin_memory().numpy()
    exp = {k[4:]: v for k, v in f.items() if k.startswith("out_")}
    tuned = dev.autotune_host(rays)
    assert 0 <= tuned["shape"] < accel.TRACE_SHAPES and min(tuned["times_ms"]) > 0
    check_closest(dev.intersect_host(rays), None, exp)
    for shape in (0, 8, 12):
        dev.set_host_trace_shape(shape)
        check_closest(dev.intersect_host(rays), None, exp)
        assert np.array_equal(dev.intersect_host(rays, any_hit=True).astype(bool), exp["hit"].astype(bool))
    dev.set_host_trace_shape(-1)
    with pytest.raises(Exception):
        dev.set_host_trace_shape(accel.TRACE_SHAPES)


def test_probe_matches_golden(cuda):
    import torch

    f = load("probe_layers")
    g = geometry(f)
    dev = accel.DeviceAccelerator(g, accel.build_bvh(g))
    hits, inst, counts, ex = dev.probe(torch.from_numpy(f["rays"]).to(cuda), torch.from_numpy(f["targets"]).to(cuda))
    dev.check()
    counts = counts.cpu().numpy()
    hits = hits.cpu().numpy()
    assert np.array_equal(counts, f["out_count"])
    assert np.array_equal(ex.cpu().numpy(), f["out_exhausted"])
    for i in np.nonzero(counts)[0]:
        c = counts[i]
        assert np.array_equal(bits(hits[i, :c, 0]), bits(f["out_t"][i, :c]))
        want = f["out_triangle_index"][i, :c]
        ids = accel.hit_ids(hits[i, :c])
        assert np.array_equal(np.where(want >= 0, ids, -1), want)


def test_probe_two_level_matches_oracle(cuda):
    import torch

    f = load("trace_two_level")
    g = geometry(f)
    tl = accel.build_two_level_bvh(g)
    rng = np.random.default_rng(5)
    rays = scenes.incoherent_rays(2000, seed=41, box=20.0)
    rays[:, 7] = 40.0
    targets = np.zeros((2000, 4), np.int32)
    targets[:, 0] = rng.integers(0, 2, 2000)
    targets[:, 1] = rng.integers(-1, 7, 2000)
    targets[:, 2] = -1
    hits, inst, counts, ex = accel.DeviceAccelerator(g, tl).probe(torch.from_numpy(rays).to(cuda),
                                                                  torch.from_numpy(targets).to(cuda))
    ohits, ocounts, oex = oracle.OracleScene(g, tl).probe(rays, targets)
    assert np.array_equal(counts.cpu().numpy(), ocounts)
    assert np.array_equal(ex.cpu().numpy(), oex)
    hits = hits.cpu().numpy()
    inst = inst.cpu().numpy()
    for i in np.nonzero(ocounts)[0]:
        c = ocounts[i]
        assert np.array_equal(bits(hits[i, :c, 0]), bits(ohits["t"][i, :c]))
        assert np.array_equal(inst[i, :c], ohits["instance"][i, :c])
    assert ocounts.sum() > 20


@pytest.fixture(scope="module")
def full_set():
    g = scenes.traversal_scene()
    return g, accel.build_bvh(g)


@pytest.mark.parametrize("kind", ["incoherent", "coherent", "shadow"])
def test_full_traversal_set_bit_exact(cuda, full_set, kind):
    """2,097,152 triangles; 2M-ray subsamples of each ray set vs the oracle."""
    import torch

    g, b = full_set
    if kind == "incoherent":
        rays = scenes.incoherent_rays(2_000_000, seed=2)
    elif kind == "coherent":
        rays = scenes.coherent_rays(1414, 1414)
    else:
        rays = scenes.shadow_rays(2_000_000, seed=3)
    dev = accel.DeviceAccelerator(g, b)
    rd = torch.from_numpy(rays).to(cuda)
    exp, st = oracle.OracleScene(g, b).trace(rays, stats=True)
    if kind == "shadow":
        occ = dev.intersect(rd, any_hit=True).cpu().numpy()
        assert np.array_equal(occ.astype(bool), exp["hit"].astype(bool))
    else:
        hits = dev.intersect(rd)
        check_closest(hits, None, exp)
        gst = dev.trace_stats(rd).cpu().numpy()
        assert np.array_equal(gst[0], st[0]) and np.array_equal(gst[1], st[1])
    dev.check()


@pytest.fixture(scope="module")
def live_full_set(ref):
    """The traversal set's BVH as the compiled reference's own BuildBvh made it."""
    g = scenes.traversal_scene()
    rs = ref.RefScene(g)
    nodes, pi, prims, depth = rs.flat_bvh()
    return g, rs, RenderBvh(nodes, pi, prims, depth)


@pytest.mark.parametrize("kind", ["incoherent", "coherent", "shadow"])
def test_full_set_against_live_reference(cuda, live_full_set, kind):
    """Every one of the 7,997,584 rays of a set, traced on the device over the
    reference's own BVH and by the compiled reference's IntersectBvh
    (src/accel/bvh_traversal.cpp:253-345) on the host: ids, t, u and v
    bit-identical and per-ray node and triangle test counts equal; for the
    shadow set, occlusion equals IntersectBvh(ray, t_min, t_max).hit."""
    import torch

    g, rs, b = live_full_set
    rays = {"incoherent": lambda: scenes.incoherent_rays(seed=2), "coherent": lambda: scenes.coherent_rays(),
            "shadow": lambda: scenes.shadow_rays(seed=3)}[kind]()
    assert rays.shape[0] == 2828 * 2828
    exp = rs.trace(rays)
    dev = accel.DeviceAccelerator(g, b)
    rd = torch.from_numpy(rays).to(cuda)
    if kind == "shadow":
        occ = dev.intersect(rd, any_hit=True).cpu().numpy()
        assert np.array_equal(occ.astype(bool), exp["hit"].astype(bool))
    else:
        check_closest(dev.intersect(rd), None, exp)
        gst = dev.trace_stats(rd).cpu().numpy()
        assert np.array_equal(gst[0], exp["node_tests"]) and np.array_equal(gst[1], exp["triangle_tests"])
    dev.check()


def test_full_size_properties(cuda, full_set):
    """At the full 7,997,584-ray size: closest-hit t never exceeds the any-hit
    t_max window when occluded, and any-hit == (closest hit exists)."""
    import torch

    g, b = full_set
    rays = torch.from_numpy(scenes.incoherent_rays()).to(cuda)
    dev = accel.DeviceAccelerator(g, b)
    hits = dev.intersect(rays)
    occ = dev.intersect(rays, any_hit=True)
    dev.check()
    ids = hits[:, 1].contiguous().view(torch.int32)
    assert torch.equal(occ.bool(), ids != -1)
    # determinism: a second launch is bit-identical
    hits2 = dev.intersect(rays)
    assert torch.equal(hits.view(torch.int32), hits2.view(torch.int32))


def test_empty_bvh_and_degenerate_inputs(cuda):
    import torch

    g = SceneGeometry.from_meshes([])
    dev = accel.DeviceAccelerator(g, accel.build_bvh(g))
    rays = torch.from_numpy(scenes.incoherent_rays(1000, seed=1)).to(cuda)
    hits = dev.intersect(rays).cpu().numpy()
    assert (accel.hit_ids(hits) == -1).all()
    assert np.isinf(hits[:, 0]).all()
    st = dev.trace_stats(rays).cpu().numpy()
    assert (st == 0).all()
    # zero rays is a no-op
    dev.intersect(rays[:0])
    dev.check()


def chain_bvh(m):
    """A hand-built chain BVH over m triangles spaced along x (any valid
    RenderBvh is accepted by the drop-in boundary): node 2k is interior with
    its left child a leaf holding triangle k and its right child the rest of
    the chain. Depth m, so a ray travelling towards -x pushes one entry per
    level."""
    meshes = []
    for i in range(m):
        x = np.float32(i)
        meshes.append((np.array([[x, -1, -1], [x, 1, -1], [x, 0, 1]], np.float32), [[0, 1, 2]]))
    g = SceneGeometry.from_meshes(meshes)
    from yaoray_b200 import _lib
    nodes = np.zeros(2 * m - 1, _lib.NODE_DTYPE)
    prims = np.zeros(m, _lib.BVH_PRIM_DTYPE)
    prims["kind"] = 0
    prims["mesh_primitive"] = np.arange(m)
    prims["sphere"] = -1
    prims["local_triangle"] = 0
    prims["flat_triangle_index"] = np.arange(m)
    for k in range(m):
        leaf = 2 * k + 1 if k < m - 1 else 2 * k
        nodes[leaf]["bounds_min"] = (k, -1, -1)
        nodes[leaf]["bounds_max"] = (k, 1, 1)
        nodes[leaf]["payload_offset"] = k
        nodes[leaf]["primitive_count"] = 1
        if k < m - 1:
            nodes[2 * k]["bounds_min"] = (k, -1, -1)
            nodes[2 * k]["bounds_max"] = (m - 1, 1, 1)
            nodes[2 * k]["payload_offset"] = 2 * k + 2
            nodes[2 * k]["primitive_count"] = 0
    return g, RenderBvh(nodes, np.arange(m, dtype=np.int32), prims, m)


def test_deep_bvh_uses_the_deep_stack_kernel(cuda):
    """A 150-level chain (deeper than the 64-entry kernel) traversed towards
    -x spills the stack into local memory; results match the oracle."""
    import torch

    g, b = chain_bvh(150)
    rng = np.random.default_rng(9)
    rays = np.zeros((4000, 8), np.float32)
    rays[:, 0] = 200.0
    rays[:, 1:3] = rng.uniform(-0.5, 0.5, (4000, 2))
    rays[:, 3] = 1e-5
    d = np.stack([-np.ones(4000), rng.normal(0, 0.003, 4000), rng.normal(0, 0.003, 4000)], 1)
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 7] = rng.choice([np.inf, 120.0, 1e30], 4000)
    dev = accel.DeviceAccelerator(g, b)
    hits = dev.intersect(torch.from_numpy(rays).to(cuda))
    dev.check()
    exp, st = oracle.OracleScene(g, b).trace(rays)
    check_closest(hits, None, exp)
    assert st[0].max() > 200


def test_too_deep_bvh_is_rejected_not_run():
    from yaoray_b200 import YrcError

    g, b = chain_bvh(300)
    with pytest.raises(YrcError, match="too deep"):
        accel.DeviceAccelerator(g, b)


def test_every_launch_shape_is_bit_identical(cuda, full_set):
    """The autotuner may pick any compiled launch shape: all must produce the
    same bits for closest and any hit."""
    import torch

    g, b = full_set
    dev = accel.DeviceAccelerator(g, b)
    rays = torch.from_numpy(scenes.incoherent_rays(500_000, seed=77)).to(cuda)
    base_hits = dev.intersect(rays).clone()
    base_occ = dev.intersect(rays, any_hit=True).clone()
    for shape in range(accel.TRACE_SHAPES):
        dev.set_trace_shape(shape)
        dev.set_trace_shape(shape, any_hit=True)
        assert torch.equal(dev.intersect(rays).view(torch.int32), base_hits.view(torch.int32)), shape
        assert torch.equal(dev.intersect(rays, any_hit=True), base_occ), shape
    tuned = dev.autotune(rays)
    assert 0 <= tuned["shape"] < accel.TRACE_SHAPES and min(tuned["times_ms"]) > 0
    dev.check()


def test_four_wide_traversal_matches_binary(cuda, full_set):
    """The four-wide copy of a triangle-only BVH gives the binary traversal's
    hits bit for bit (closest and any hit, every launch shape), as the
    reference pins for its BVH4; BVHs with spheres have no four-wide copy."""
    import torch

    g, b = full_set
    dev = accel.DeviceAccelerator(g, b)
    assert not dev.wide  # opt-in
    rays = torch.from_numpy(np.concatenate([scenes.incoherent_rays(400_000, seed=91),
                                            scenes.coherent_rays(400, 400),
                                            scenes.shadow_rays(200_000, seed=92)])).to(cuda)
    bin_hits = dev.intersect(rays).clone()
    bin_occ = dev.intersect(rays, any_hit=True).clone()
    dev.set_wide(True)
    assert dev.wide
    wide_hits = dev.intersect(rays)
    wide_occ = dev.intersect(rays, any_hit=True)
    assert torch.equal(wide_hits.view(torch.int32), bin_hits.view(torch.int32))
    assert torch.equal(wide_occ, bin_occ)
    for shape in range(accel.TRACE_SHAPES):
        dev.set_trace_shape(shape)
        assert torch.equal(dev.intersect(rays).view(torch.int32), bin_hits.view(torch.int32)), shape
    dev.check()
    gs = geometry(load("trace_spheres"))
    assert gs.spheres.size > 0
    with pytest.raises(Exception):
        accel.DeviceAccelerator(gs, accel.build_bvh(gs)).set_wide(True)


def test_ray_order_keeps_every_hit(cuda, full_set):
    """Reordering the rays before a trace (both key kinds, several key
    sizes) changes only which lanes share a warp: closest and any hits are
    those of the unordered trace, bit for bit, for incoherent, coherent
    (many rays per key bin) and shadow rays, and the timing entry point
    reports both stages."""
    import torch

    g, b = full_set
    dev = accel.DeviceAccelerator(g, b)
    assert dev.ray_order == "off"
    rays = torch.from_numpy(np.concatenate([scenes.incoherent_rays(300_000, seed=93),
                                            scenes.coherent_rays(400, 400),
                                            scenes.shadow_rays(200_000, seed=94)])).to(cuda)
    ref_hits = dev.intersect(rays).clone()
    ref_occ = dev.intersect(rays, any_hit=True).clone()
    dev.set_timing(True)
    for mode, bits, length in (("direction", 0, 0.05), ("direction", 8, 0.05), ("two-point", 19, 0.15),
                               ("two-point", 24, 0.02)):
        dev.set_ray_order(mode, bits, length)
        assert dev.ray_order == mode
        hits = dev.intersect(rays)
        order_ms, trace_ms = dev.last_timing()
        assert order_ms > 0.0 and trace_ms > 0.0
        assert torch.equal(hits.view(torch.int32), ref_hits.view(torch.int32)), (mode, bits)
        assert torch.equal(dev.intersect(rays, any_hit=True), ref_occ), (mode, bits)
    dev.set_ray_order("off")
    dev.intersect(rays)
    assert dev.last_timing()[0] == 0.0
    dev.check()
    with pytest.raises(Exception):
        dev.set_ray_order("two-point", 25, 0.1)


@pytest.mark.parametrize("name", ["trace_two_level", "trace_spheres"])
def test_every_launch_shape_matches_golden(cuda, name):
    """Every compiled launch shape, two-level and sphere BVHs included, gives
    the reference's hits (the autotuners may pick any of them)."""
    import torch

    f = load(name)
    g, b = golden_accel(f, name)
    dev = accel.DeviceAccelerator(g, b)
    rays = torch.from_numpy(f["rays"]).to(cuda)
    exp = {k[4:]: v for k, v in f.items() if k.startswith("out_")}
    for shape in range(accel.TRACE_SHAPES):
        dev.set_trace_shape(shape)
        dev.set_trace_shape(shape, any_hit=True)
        inst = torch.empty(rays.shape[0], dtype=torch.int32, device=cuda)
        hits = dev.intersect(rays, instances=inst)
        occ = dev.intersect(rays, any_hit=True)
        check_closest(hits, inst, exp, exp["instance"])
        assert np.array_equal(occ.cpu().numpy().astype(bool), exp["hit"].astype(bool)), shape
    dev.check()
