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
