"""What the trained radiance cache gains: on the instanced scene at test size
(radiance clamp 20 for every render), a cache trained online for a few
batches lets the path tracer end paths early; at equal samples per pixel its
image must be closer to a high-sample plain reference (relMSE, FP64
accumulation) than the plain render, with the image mean within 5 % of the
reference's (the cache's bias is bounded), while tracing fewer path
segments."""
import numpy as np
import pytest

from yaoray_b200 import instanced
from yaoray_b200.nrc import RadianceCache
from yaoray_b200.render import CudaBackend

pytestmark = pytest.mark.gpu
W, H, CLAMP = 200, 112, 20.0


def scene(spp, seed):
    s = instanced.scene(width=W, height=H, spp=spp, mesh_scale=0.1, instances=64, env_width=512)
    s.radiance_clamp = CLAMP
    s.seed = seed
    return s


def relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def test_trained_cache_beats_plain_at_equal_spp(cuda):
    b = CudaBackend()
    ref = np.zeros((H, W, 3), np.float64)
    for k in range(4):
        p = b.prepare(scene(128, 1000 + k))
        r = b.render(p)
        assert r.ok, r.error
        ref += r.linear()
        p.close()
    ref /= 4
    p = b.prepare(scene(4, 7))
    plain = b.render(p)
    p.close()
    base = scene(1, 0)
    lo = base.geometry.positions.min(0)
    extent = float((base.geometry.positions.max(0) - lo).max())
    cache = RadianceCache(lo, extent, seed=1)
    warm = b.prepare(scene(2, 99))
    warm.set_radiance_cache(cache, spread_threshold=0.001, train_steps=4)
    for _ in range(8):
        assert b.render(warm).ok
    warm.close()
    p = b.prepare(scene(4, 7))
    p.set_radiance_cache(cache, spread_threshold=0.001)
    cached = b.render(p)
    assert cached.ok, cached.error
    cache.check()
    assert cached.stats["cache_queries"] > 0 and cached.stats["cache_records"] > 0
    e_plain, e_cached = relmse(plain.linear(), ref), relmse(cached.linear(), ref)
    assert e_cached < 0.9 * e_plain, (e_cached, e_plain)
    assert abs(cached.linear().mean() / ref.mean() - 1) < 0.05
    assert cached.stats["rays_traced"] < plain.stats["rays_traced"]
    # detaching restores the plain tracer bit for bit
    p.set_radiance_cache(None)
    again = b.render(p)
    assert again.film.tobytes() == plain.film.tobytes()
    cache.close()
