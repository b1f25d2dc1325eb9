"""Coated (layered) materials in the path tracer against the reference CPU
backend, pixel by pixel.

The layered BSDF draws from the path's PCG32 stream. The reference draws for
an emissive next event only when its shadow ray came back visible, evaluates
the analytic and environment samples before their shadow rays, draws the
environment pdf after its ray, and samples the continuation after all of
that (EstimateDirectLight, src/integrators/path_direct_lighting.cpp:115-283;
IntegratePathSample, src/integrators/path_integrator.cpp:93-192). The device
keeps that order (DeferLayeredVertex, LayeredNeeKernel,
LayeredContinueKernel), so a render with the same seed follows the
reference's paths: each pixel agrees with the reference to rounding, except
where a walk takes another branch because CUDA's expf or sinf/cosf rounded
apart from glibc's (a draw compared with a Fresnel value, a direction a few
ulps apart that hits another surface). With the draws in another order, the
coated pixels whose emissive shadow ray is occluded would follow unrelated
paths.

Scene: the Cornell box with the floor and both boxes coated diffuse, lit by
its area light, a point, a spot and a distant light, and a sky seen through
its open front. Stated bound: at max depth 2 and 3, the share of pixels whose
beauty agrees with the same-seed reference within a relative 1e-3 is at least
the bound in AGREE (measured values in its comment), while two reference
renders with different seeds agree on about 6 % (pixels that see only
the light).
"""
import numpy as np
import pytest

from yaoray_b200 import cornell, instanced
from yaoray_b200.render import COATED_DIFFUSE, CudaBackend, EnvironmentMap, default_material

pytestmark = pytest.mark.gpu

AGREE = {2: 0.99, 3: 0.99}  # measured on a B200: 1.0000 at both depths


def coated_scene(depth, seed=0, size=64, spp=4):
    s = cornell.analytic_scene(size, size, spp, depth)
    coat = default_material(kind=COATED_DIFFUSE, reflectance=(0.7, 0.6, 0.5), coat_thickness=0.01,
                            coat_absorption=(0.3, 0.1, 0.05))
    s.materials = np.concatenate([s.materials, coat[None]])
    k = len(s.materials) - 1
    for prim in (0, 5, 6):  # floor, short box, tall box
        s.geometry.primitives[prim]["material_index"] = k
    env = EnvironmentMap(active=True, radiance=(1.0, 1.0, 1.0), strength=0.5, rotation=0.0,
                         texels=instanced.hdri(128, 64))
    env.build_distribution()
    s.environment = env
    s.radiance_clamp = 20.0
    s.seed = seed
    return s


def _linear(film):
    s = film["samples"].astype(np.float64)
    out = np.zeros(film["sum"].shape, np.float64)
    nz = s > 0
    out[nz] = film["sum"][nz] / s[nz][..., None]
    return out


def _agree(a, b):
    rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-2)
    return float((rel.max(-1) <= 1e-3).mean())


@pytest.mark.parametrize("depth", [2, 3])
def test_coated_render_follows_reference_paths(cuda, ref, depth):
    scene = coated_scene(depth)
    res = CudaBackend().render(CudaBackend().prepare(scene))
    assert res.ok, res.error
    cpu, cpu_stats, _ = ref.RefJob.from_scene(scene).render()
    other, _, _ = ref.RefJob.from_scene(coated_scene(depth, seed=7)).render()
    g, c, o = _linear(res.film), _linear(cpu.reshape(res.film.shape)), _linear(other.reshape(res.film.shape))
    agree, seed_agree = _agree(g, c), _agree(o, c)
    print(f"\ncoated depth {depth}: agree {agree:.4f}, seed-to-seed {seed_agree:.4f}, "
          f"shadow rays {res.stats['shadow_rays']} vs {cpu_stats['shadow_rays']}, "
          f"occluded {res.stats['occluded_shadow_rays']} vs {cpu_stats['occluded_shadow_rays']}")
    assert seed_agree < 0.1
    assert agree >= AGREE[depth], (agree, seed_agree)
    # the same shadow rays traced and found occluded (measured: identical counts)
    assert abs(res.stats["shadow_rays"] / cpu_stats["shadow_rays"] - 1) < 1e-3
    assert abs(res.stats["occluded_shadow_rays"] / cpu_stats["occluded_shadow_rays"] - 1) < 1e-3
