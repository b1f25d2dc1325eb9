"""Batched uneven render jobs on the device: concurrent rendering from
worker threads (one stream per job) gives the same films as one-at-a-time
rendering for jobs without a radiance cache, and every job completes."""
import numpy as np
import pytest

from yaoray_b200 import batch

pytestmark = pytest.mark.gpu


def test_concurrent_matches_sequential():
    jobs = batch.job_set(8, seed=11, spp_scale=1 / 64, max_triangles=120_000)
    runner = batch.JobRunner(keep_films=True)
    try:
        runner.prepare(jobs)
        seq = runner.run_sequential(jobs)
        assert all(j.ok for j in jobs), [j.error for j in jobs if not j.ok]
        films = {j.name: j.film.copy() for j in jobs}
        conc = runner.run_concurrent(jobs, concurrency=4)
        assert all(j.ok for j in jobs), [j.error for j in jobs if not j.ok]
        assert conc.samples == seq.samples == sum(j.scene.width * j.scene.height * j.scene.spp for j in jobs)
        assert conc.peak_concurrency > 1
        for j in jobs:
            f = j.film
            assert np.isfinite(f["sum"]).all()
            assert (f["samples"] == j.scene.spp).all()
            if not j.use_cache:
                # Deterministic per job: the other jobs on other streams change nothing.
                assert np.array_equal(f["sum"], films[j.name]["sum"]), j.name
            assert f["sum"].mean() > 0
    finally:
        runner.close(jobs)


def test_shared_launch_matches_single_renders():
    """yrc_render_many: one graph launch per step for all unfinished jobs;
    films equal one-at-a-time renders for the jobs without a cache."""
    jobs = batch.job_set(6, seed=13, spp_scale=1 / 64, max_triangles=100_000)
    runner = batch.JobRunner(keep_films=True)
    try:
        runner.prepare(jobs)
        runner.run_sequential(jobs)
        films = {j.name: j.film.copy() for j in jobs}
        res = runner.run_shared_launch(jobs, concurrency=6)
        assert all(j.ok for j in jobs), [j.error for j in jobs if not j.ok]
        assert res.peak_concurrency > 1
        for j in jobs:
            assert (j.film["samples"] == j.scene.spp).all()
            if not j.use_cache:
                assert j.film.tobytes() == films[j.name].tobytes(), j.name
    finally:
        runner.close(jobs)


def test_shared_launch_rejects_bad_groups():
    """yrc_render_many refuses a scene given twice and two scenes that share
    one radiance cache (their training steps would race), with an error."""
    from yaoray_b200.nrc import RadianceCache
    from yaoray_b200.render import CudaBackend

    jobs = batch.job_set(2, seed=17, spp_scale=1 / 64, max_triangles=30_000)
    b = CudaBackend()
    p0, p1 = b.prepare(jobs[0].scene), b.prepare(jobs[1].scene)
    try:
        twice = b.render_many([p0, p0])
        assert not twice[0].ok and "twice" in twice[0].error
        lo = jobs[0].scene.geometry.positions.min(0)
        cache = RadianceCache(lo, 200.0, seed=1)
        p0.set_radiance_cache(cache)
        p1.set_radiance_cache(cache)
        shared = b.render_many([p0, p1])
        assert not shared[0].ok and "share a radiance cache" in shared[0].error
        p1.set_radiance_cache(None)
        ok = b.render_many([p0, p1])
        assert ok[0].ok and ok[1].ok
        p0.set_radiance_cache(None)
        cache.close()
    finally:
        p0.close()
        p1.close()


def test_shared_launch_renders_every_scene_kind():
    """The stages that only some scenes need (texture stage, cut-out skip
    loop, exact shadow loop, measured BRDFs, analytic lights with the light
    tree) inside one shared launch: films equal one-at-a-time renders."""
    from yaoray_b200 import cornell
    from yaoray_b200.render import CudaBackend

    scenes = [cornell.textured_scene(48, 48, 8, 6), cornell.cutout_scene(48, 48, 8, 6),
              cornell.instanced_cutout_scene(48, 48, 8, 6), cornell.measured_scene(48, 48, 8, 6),
              cornell.analytic_scene(48, 48, 8, 6, many=True), cornell.scene(48, 48, 8, 6)]
    b = CudaBackend()
    prepared = [b.prepare(s) for s in scenes]
    singles = [b.render(p) for p in prepared]
    many = b.render_many(prepared)
    for k, (one, shared) in enumerate(zip(singles, many)):
        assert one.ok and shared.ok, (k, one.error, shared.error)
        assert shared.film.tobytes() == one.film.tobytes(), k


def test_pooled_launch_matches_single_renders():
    """yrc_render_pooled: per bounce one persistent traversal launch serves
    the extend rays of every unfinished job and one their shadow rays; the
    films equal one-at-a-time renders byte for byte for the jobs without a
    cache (a ray's hit does not depend on which launch traced it)."""
    jobs = batch.job_set(6, seed=13, spp_scale=1 / 64, max_triangles=100_000)
    runner = batch.JobRunner(keep_films=True)
    try:
        runner.prepare(jobs)
        runner.run_sequential(jobs)
        films = {j.name: j.film.copy() for j in jobs}
        res = runner.run_shared_launch(jobs, concurrency=6, pooled=True)
        assert all(j.ok for j in jobs), [j.error for j in jobs if not j.ok]
        assert res.peak_concurrency > 1
        for j in jobs:
            assert (j.film["samples"] == j.scene.spp).all()
            if not j.use_cache:
                assert j.film.tobytes() == films[j.name].tobytes(), j.name
    finally:
        runner.close(jobs)


def test_pooled_launch_renders_every_scene_kind():
    """Pooled launches over scenes of every kind: flat and two-level BVHs
    (one pooled launch per kind), exact-loop shadows (traced per scene),
    transmittance and any-hit shadows (pooled); films equal one-at-a-time
    renders."""
    from yaoray_b200 import cornell
    from yaoray_b200.render import CudaBackend

    scenes = [cornell.textured_scene(48, 48, 8, 6), cornell.cutout_scene(48, 48, 8, 6),
              cornell.instanced_cutout_scene(48, 48, 8, 6), cornell.measured_scene(48, 48, 8, 6),
              cornell.analytic_scene(48, 48, 8, 6, many=True), cornell.scene(48, 48, 8, 6),
              cornell.scene(32, 40, 4, 3)]
    b = CudaBackend()
    prepared = [b.prepare(s) for s in scenes]
    singles = [b.render(p) for p in prepared]
    pooled = b.render_many(prepared, pooled=True)
    for k, (one, shared) in enumerate(zip(singles, pooled)):
        assert one.ok and shared.ok, (k, one.error, shared.error)
        assert shared.film.tobytes() == one.film.tobytes(), k
        assert shared.stats["rays_traced"] == one.stats["rays_traced"], k
        assert shared.stats["occluded_shadow_rays"] == one.stats["occluded_shadow_rays"], k
