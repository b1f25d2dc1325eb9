"""Render autotuner: the queue capacity changes how many passes a batch
holds, never the film (samples are a function of pixel and sample index and
the film adds them in pass order); the autotuner picks one of its candidates
and later renders use it."""
import numpy as np
import pytest

from yaoray_b200 import accel, batch, cornell
from yaoray_b200.render import CudaBackend

pytestmark = pytest.mark.gpu


def test_film_independent_of_capacity():
    b = CudaBackend()
    scene = cornell.scene(width=64, height=48, spp=16)
    p = b.prepare(scene)
    films = []
    for cap in (0, 64 * 48, 64 * 48 * 4, 64 * 48 * 16):
        p.set_capacity(cap)
        r = b.render(p)
        assert r.ok, r.error
        films.append(r.film.copy())
    assert p.capacity == 64 * 48 * 16
    p.close()
    for f in films[1:]:
        assert f.tobytes() == films[0].tobytes()


def test_autotune_chooses_a_candidate_and_keeps_it():
    b = CudaBackend()
    job = batch.job_set(2, seed=3, spp_scale=1 / 16, max_triangles=60_000)[0]
    p = b.prepare(job.scene)
    ref = b.render(p)
    assert ref.ok, ref.error
    t = p.autotune()
    pixels = job.scene.width * job.scene.height
    assert t["capacity"] % pixels == 0 and pixels <= t["capacity"] <= pixels * min(job.scene.spp, 64)
    assert 0 <= t["trace_shape"] < accel.TRACE_SHAPES and t["candidates"] >= 2 and t["seconds_per_sample"] > 0
    assert p.capacity == t["capacity"]
    again = b.render(p)
    assert again.ok, again.error
    assert again.film.tobytes() == ref.film.tobytes()
    p.close()


@pytest.mark.parametrize("make", [lambda: batch.job_set(2, seed=5, spp_scale=1 / 64, max_triangles=60_000)[0].scene,
                                  lambda: cornell.instanced_cutout_scene(48, 48, 8, 6)],
                         ids=["flat-glass-subsurface", "two-level-cutout"])
def test_film_independent_of_launch_shape(make):
    """Every launch shape the render autotuner may choose (leaf batching in
    the extend, shadow-transmittance and any-hit traversals included) gives
    the film of the default shape byte for byte, on a flat scene with glass,
    coated and subsurface materials and on a two-level scene with cut-outs."""
    b = CudaBackend()
    scene = make()
    p = b.prepare(scene)
    cap = scene.width * scene.height * min(scene.spp, 4)
    films = []
    for shape in range(accel.TRACE_SHAPES):
        p.set_tuning({"capacity": cap, "trace_shape": shape})
        r = b.render(p)
        assert r.ok, (shape, r.error)
        films.append(r.film.copy())
    p.close()
    for shape, f in enumerate(films[1:], 1):
        assert f.tobytes() == films[0].tobytes(), shape
