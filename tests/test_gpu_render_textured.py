"""Textured shading parity: the textured Cornell box (reflectance textures
under every filter and wrap mode, a tangent-space normal map with per-vertex
tangents) through the CUDA backend and the reference CpuBackend on the same
IR.

First-hit depth and normal sums are bit-identical (the normal map is looked
up bilinearly, which is bit-exact). First-hit albedo sums include trilinear
and EWA lookups, whose level of detail goes through log2f (the host C
library's last bit can differ from the device's correctly rounded log2), so
they must agree within a relative 1e-5 and be bit-identical in at least 99 %
of pixels. The beauty film obeys the same relMSE bound as the untextured
renders: below 0.25x the relMSE between two CPU seeds, image mean within 1 %.
"""
import numpy as np
import pytest

from yaoray_b200 import cornell
from yaoray_b200.render import CudaBackend

pytestmark = pytest.mark.gpu


def linear(film):
    s = film["samples"].astype(np.float64)
    out = np.zeros(film["sum"].shape, np.float64)
    nz = s > 0
    out[nz] = film["sum"][nz] / s[nz][:, None]
    return out


def relmse(a, b):
    return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))


def render_pair(ref, make):
    scene = make(0)
    backend = CudaBackend()
    res = backend.render(backend.prepare(scene))
    assert res.ok, res.error
    cpu_film, cpu_stats, _ = ref.RefJob.from_scene(scene).render()
    cpu2, _, _ = ref.RefJob.from_scene(make(12345)).render()
    return res, cpu_film, cpu_stats, cpu2


def check_aovs(res, cpu_film):
    assert np.array_equal(res.film["samples"], cpu_film["samples"])
    assert np.array_equal(res.film["aov_samples"], cpu_film["aov_samples"])
    assert res.film["depth_sum"].tobytes() == cpu_film["depth_sum"].tobytes()
    assert res.film["normal_sum"].tobytes() == cpu_film["normal_sum"].tobytes()
    a, b = res.film["albedo_sum"], cpu_film["albedo_sum"]
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6)
    same = np.all(a.view(np.uint32) == b.view(np.uint32), axis=-1)
    assert same.mean() >= 0.99, same.mean()


def test_textured_cornell_matches_reference_cpu(cuda, ref):
    def make(seed):
        s = cornell.textured_scene(96, 96, 64, 8)
        s.seed = seed
        return s

    res, cpu_film, cpu_stats, cpu2 = render_pair(ref, make)
    check_aovs(res, cpu_film)
    g, c, c2 = linear(res.film), linear(cpu_film), linear(cpu2)
    noise = relmse(c2, c)
    err = relmse(g, c)
    assert err < 0.25 * noise, (err, noise)
    assert abs(g.mean() / c.mean() - 1.0) < 0.01
    assert res.bad_samples == 0
    assert abs(res.stats["rays_traced"] / cpu_stats["rays_traced"] - 1) < 0.02
    assert abs(res.stats["shadow_rays"] / cpu_stats["shadow_rays"] - 1) < 0.02


def test_textures_change_the_render_and_share_pyramids(cuda):
    """Textures are applied (the albedo AOV differs from the untextured box)
    and identical images share one pyramid on the device."""
    plain = CudaBackend()
    a = plain.render(plain.prepare(cornell.scene(48, 48, 4, 4)))
    s = cornell.textured_scene(48, 48, 4, 4)
    b = plain.render(plain.prepare(s))
    assert a.ok and b.ok
    assert not np.array_equal(a.film["albedo_sum"], b.film["albedo_sum"])
    assert not np.array_equal(a.film["normal_sum"], b.film["normal_sum"])
    one = plain.prepare(s).device_bytes
    s.textures = s.textures + [s.textures[0], s.textures[0]]  # two more copies of the floor's image
    assert plain.prepare(s).device_bytes - one < 4096


def test_cutout_scene_matches_reference_cpu(cuda, ref):
    """Alpha: a screen with an alpha texture cutting round holes in front
    of the boxes, a pane with constant alpha 0.2 under the light (every ray
    skips it, shadow rays included), and thin glass with a textured
    reflectance (shadow rays take its textured transmittance). The skip
    loops re-trace from just past each cut-out hit as the reference does,
    so first hits, and with them the depth and normal sums, stay
    bit-identical."""
    def make(seed):
        s = cornell.cutout_scene(96, 96, 64, 8)
        s.seed = seed
        return s

    res, cpu_film, cpu_stats, cpu2 = render_pair(ref, make)
    check_aovs(res, cpu_film)
    g, c, c2 = linear(res.film), linear(cpu_film), linear(cpu2)
    noise = relmse(c2, c)
    err = relmse(g, c)
    assert err < 0.25 * noise, (err, noise)
    assert abs(g.mean() / c.mean() - 1.0) < 0.01
    assert res.bad_samples == 0
    assert abs(res.stats["rays_traced"] / cpu_stats["rays_traced"] - 1) < 0.02
    assert abs(res.stats["shadow_rays"] / cpu_stats["shadow_rays"] - 1) < 0.02
    assert abs(res.stats["occluded_shadow_rays"] / cpu_stats["occluded_shadow_rays"] - 1) < 0.03


def test_instanced_cutout_scene_matches_reference_cpu(cuda, ref):
    """The cut-out scene as a two-level scene: the normal map on a mirrored
    instance (negative determinant: the tangent frame flips), the alpha
    screen under a tilt and a translation (footprints from transformed
    triangles), every other primitive under an identity instance."""
    def make(seed):
        s = cornell.instanced_cutout_scene(96, 96, 64, 8)
        s.seed = seed
        return s

    res, cpu_film, cpu_stats, cpu2 = render_pair(ref, make)
    check_aovs(res, cpu_film)
    g, c, c2 = linear(res.film), linear(cpu_film), linear(cpu2)
    noise = relmse(c2, c)
    err = relmse(g, c)
    assert err < 0.25 * noise, (err, noise)
    assert abs(g.mean() / c.mean() - 1.0) < 0.01
    assert res.bad_samples == 0
    assert abs(res.stats["rays_traced"] / cpu_stats["rays_traced"] - 1) < 0.02


@pytest.mark.parametrize("many", [False, True])
def test_analytic_lights_match_reference_cpu(cuda, ref, many):
    """Point, spot and distant lights (many=False: power alias selection;
    many=True: twelve local lights, light-tree selection by power over
    distance) together with the area light."""
    def make(seed):
        s = cornell.analytic_scene(96, 96, 64, 8, many=many)
        s.seed = seed
        return s

    res, cpu_film, cpu_stats, cpu2 = render_pair(ref, make)
    g, c, c2 = linear(res.film), linear(cpu_film), linear(cpu2)
    noise = relmse(c2, c)
    err = relmse(g, c)
    assert err < 0.25 * noise, (err, noise)
    assert abs(g.mean() / c.mean() - 1.0) < 0.01
    assert res.film["depth_sum"].tobytes() == cpu_film["depth_sum"].tobytes()
    assert abs(res.stats["shadow_rays"] / cpu_stats["shadow_rays"] - 1) < 0.02
    assert abs(res.stats["occluded_shadow_rays"] / cpu_stats["occluded_shadow_rays"] - 1) < 0.03
