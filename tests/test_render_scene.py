"""CPU checks of the render-side host logic: the Cornell scene generator
builds the same RenderSceneIR the reference's PBRT frontend compiles from the
generated file; the host alias-table and environment-distribution builders
reproduce the reference's tables."""
import numpy as np
import pytest

from yaoray_b200 import cornell
from yaoray_b200.render import build_alias_table, EnvironmentMap


def test_cornell_config_shape():
    s = cornell.scene()
    assert s.geometry.triangle_count == 36  # 34 scene triangles + the 2-triangle light
    assert (s.width, s.height, s.spp, s.max_depth, s.seed) == (256, 256, 64, 8, 0)
    assert s.emissive.size == 1 and tuple(s.emissive[0]["radiance"]) == (17.0, 12.0, 4.0)
    lx = cornell.shapes()[-1][1]
    assert abs((lx[2][0] - lx[0][0]) - 1.3) < 1e-6 and abs((lx[1][2] - lx[0][2]) - 1.05) < 1e-6


def test_cornell_ir_matches_reference_frontend(ref, tmp_path):
    path = tmp_path / "cornell.pbrt"
    path.write_text(cornell.pbrt_text(96, 64, 16, 8))
    theirs = ref.RefJob.load_pbrt(path).export()
    mine = cornell.scene(96, 64, 16, 8)
    assert np.array_equal(mine.geometry.positions, theirs.geometry.positions)
    assert np.array_equal(mine.geometry.indices, theirs.geometry.indices)
    assert mine.geometry.primitives.tobytes() == theirs.geometry.primitives.tobytes()
    assert mine.materials.tobytes() == theirs.materials.tobytes()
    assert mine.emissive.tobytes() == theirs.emissive.tobytes()
    for k in ("origin", "forward", "right", "up", "fov_y_radians"):
        assert np.allclose(mine.camera[k], theirs.camera[k], atol=0, rtol=0)
    assert (mine.width, mine.height, mine.spp, mine.max_depth, mine.seed, mine.sampler) == \
        (theirs.width, theirs.height, theirs.spp, theirs.max_depth, theirs.seed, theirs.sampler)
    prob, alias, pmf = mine.emissive_power_alias()
    assert np.array_equal(prob, theirs.alias[0]) and np.array_equal(alias, theirs.alias[1])
    assert np.array_equal(pmf, theirs.alias[2])


def test_alias_table_builder_pins():
    # uniform weights: every column keeps itself with probability 1
    prob, alias, pmf = build_alias_table(np.ones(5, np.float32))
    assert np.allclose(pmf, 0.2) and np.array_equal(alias, np.arange(5)) and np.allclose(prob, 1.0)
    # zero total: uniform pmf (light_sampling.cpp:165)
    prob, alias, pmf = build_alias_table(np.zeros(3, np.float32))
    assert np.allclose(pmf, 1 / 3)
    # skewed: probabilities reconstruct the pmf
    w = np.array([1, 2, 3, 10, 0.5], np.float32)
    prob, alias, pmf = build_alias_table(w)
    recon = prob / len(w)
    for i in range(len(w)):
        recon[alias[i]] += (1 - prob[i]) / len(w)
    assert np.allclose(recon, w / w.sum(), atol=1e-6)


def test_alias_table_matches_reference(ref, tmp_path):
    """Many emitters of unequal power: the product builder's table equals the
    one PrepareLightSampling builds inside the reference."""
    rng = np.random.default_rng(3)
    s = cornell.scene(16, 16, 1, 2)
    from yaoray_b200.render import EMISSIVE_DTYPE
    em = np.zeros(40, EMISSIVE_DTYPE)
    em["primitive_index"] = 7
    em["radiance"] = rng.uniform(0, 20, (40, 3))
    em["area"] = rng.uniform(0.1, 3.0, 40)
    s.emissive = em
    s.alias = None
    mine = s.emissive_power_alias()
    theirs = ref.RefJob.from_scene(s).export().alias
    for a, b in zip(mine, theirs):
        assert np.array_equal(a, b)


def test_environment_distribution_builder():
    tex = np.zeros((8, 16, 4), np.float32)
    tex[3, 5, :3] = 10.0
    tex[..., 3] = 1.0
    env = EnvironmentMap(active=True, texels=tex)
    env.build_distribution()
    w = env.texel_weights.reshape(8, 16)
    assert w.argmax() == 3 * 16 + 5
    assert np.isclose(env.total_weight, env.row_weights.sum())
    assert np.all(np.diff(env.row_cdf) >= 0)
    # all-black: uniform fallback (environment.cpp:106-120)
    env = EnvironmentMap(active=True, texels=np.zeros((4, 4, 4), np.float32))
    env.build_distribution()
    assert env.total_weight == 16 and np.all(env.texel_weights == 1)


def test_instanced_config_shape():
    from yaoray_b200 import instanced
    s = instanced.scene(width=32, height=16, spp=1, mesh_scale=0.01, instances=40, env_width=64)
    g = s.geometry
    assert g.instances.size == 40 + 1 + 64  # instances, then identity instances of ground + emitters
    assert (g.instances["primitive"][:40] < instanced.OBJECTS).all()
    assert np.array_equal(g.instances["primitive"][40:], np.arange(instanced.OBJECTS, instanced.OBJECTS + 65))
    assert s.emissive.size == 64 and (s.emissive["area"] > 0).all()
    kinds = s.materials["kind"][: instanced.OBJECTS]
    assert [int((kinds == k).sum()) for k in (0, 1, 2, 4)] == [13, 8, 6, 5]
    # every object primitive owns its index range
    p = g.primitives
    assert (p["first_index"][1:] == p["first_index"][:-1] + p["index_count"][:-1]).all()
    assert s.environment.texels.shape == (32, 64, 4) and s.environment.total_weight > 0
    # the sun: at full resolution texels inside the 0.5 degree disk carry
    # 1e4; at any resolution the disk's power (radiance x solid angle) is kept
    import math
    sun_power = instanced.SUN_RADIANCE * 2 * math.pi * (1 - math.cos(math.radians(instanced.SUN_DIAMETER_DEG / 2)))
    for w in (256, 2048):
        t = instanced.hdri(w, w // 2)[..., 0]
        th = (np.arange(w // 2) + 0.5) * np.pi / (w // 2)
        solid = (np.pi / (w // 2)) * (2 * np.pi / w) * np.sin(th)[:, None]
        power = float((np.where(t > 2, t - 1, 0) * solid).sum())
        assert abs(power / sun_power - 1) < 0.05, (w, power, sun_power)
    assert instanced.hdri(2048, 1024)[..., 0].max() == instanced.SUN_RADIANCE


def test_instanced_full_size_counts():
    from yaoray_b200 import instanced
    ms = instanced.meshes()
    assert [t.shape[0] for _, t, _ in ms] == [50000, 75000, 100000, 249218]


def test_bssrdf_table_builder_matches_reference(ref):
    """The product's ComputeBeamDiffusionBSSRDF restatement gives the
    reference's 100 x 64 profile tables bit for bit."""
    from yaoray_b200.render import build_bssrdf_table
    for eta in (1.33, 1.5):
        mine = build_bssrdf_table(eta)
        theirs = ref.ref_bssrdf_table(0.0, eta)
        for k in mine:
            assert mine[k].tobytes() == theirs[k].tobytes(), (eta, k)
