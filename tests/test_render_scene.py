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
