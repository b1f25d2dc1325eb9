"""Batched uneven render jobs: the workload generator and the admission
scheduler (host logic, no GPU: renders are replaced by a timed stub)."""
import threading
import time

import numpy as np

from yaoray_b200 import batch


def test_job_set_shapes():
    jobs = batch.job_set(8, seed=3, spp_scale=1 / 16, max_triangles=200_000)
    assert len(jobs) == 8
    for j in jobs:
        s = j.scene
        assert s.width in batch.RESOLUTIONS and s.height == s.width
        assert 1 <= s.spp <= 1024 // 16
        assert 10_000 <= s.geometry.triangle_count <= 200_000 + 4096
        assert s.materials.size >= 5 and s.bssrdf_tables and s.radiance_clamp == 20.0
        mi = s.geometry.primitives["material_index"]
        assert mi.min() >= 0 and mi.max() < s.materials.size
    assert [j.use_cache for j in jobs] == [False, True] * 4
    again = batch.job_set(8, seed=3, spp_scale=1 / 16, max_triangles=200_000)
    assert [j.name for j in again] == [j.name for j in jobs]
    assert np.array_equal(again[5].scene.geometry.positions, jobs[5].scene.geometry.positions)


class _StubRunner(batch.JobRunner):
    """Renders by sleeping in proportion to the job's samples and records
    the summed working set of the jobs running at once."""

    def __init__(self):
        super().__init__()
        self.lock = threading.Lock()
        self.live = 0
        self.max_live = 0

    def _render(self, job):
        need = batch._working_set(job)
        with self.lock:
            self.live += need
            self.max_live = max(self.max_live, self.live)
        time.sleep(0.002 + 1e-9 * job.scene.width * job.scene.height * job.scene.spp)
        with self.lock:
            self.live -= need
        job.ok, job.samples, job.latency_s = True, job.scene.width * job.scene.height * job.scene.spp, 0.01


def test_admission_respects_budget():
    jobs = batch.job_set(12, seed=5, spp_scale=1 / 64, max_triangles=50_000)
    need = sorted(batch._working_set(j) for j in jobs)
    budget = need[-1] + need[-2] // 2  # the two largest never run together
    r = _StubRunner()
    res = r.run_concurrent(jobs, concurrency=6, budget_bytes=budget)
    assert all(j.ok for j in jobs)
    assert r.max_live <= budget
    assert res.samples == sum(j.samples for j in jobs)
    assert 1 <= res.peak_concurrency <= 6
    # With a budget that fits everything, the pool runs several jobs at once.
    r2 = _StubRunner()
    res2 = r2.run_concurrent(jobs, concurrency=6, budget_bytes=sum(need))
    assert res2.peak_concurrency > 1
    q = res2.latency_quantiles()
    assert q["p50"] == 0.01 and q["p99"] == 0.01


def test_oversized_job_runs_alone():
    jobs = batch.job_set(4, seed=9, spp_scale=1 / 64, max_triangles=50_000)
    r = _StubRunner()
    res = r.run_concurrent(jobs, concurrency=4, budget_bytes=1)
    assert all(j.ok for j in jobs) and res.peak_concurrency == 1


class _StubPrepared:
    """A prepared scene's queue-capacity rules without a device: the
    capacity is a whole number of passes between one pass and min(spp, 64)."""

    def __init__(self, scene, capacity):
        self.scene = scene
        self._cap = capacity

    @property
    def capacity(self):
        pixels = self.scene.width * self.scene.height
        return min(max(self._cap, pixels), pixels * min(self.scene.spp, 64))

    def set_tuning(self, tuning):
        self._cap = int(tuning["capacity"])


def test_fit_capacities_brings_the_working_sets_under_the_budget(monkeypatch):
    """All jobs stay resident once rendered, so preparation halves the
    largest jobs' queue capacities (whole passes, never below one) until
    every job's working memory fits the device at once."""
    jobs = batch.job_set(12, seed=5, spp_scale=1.0, max_triangles=50_000)
    for j in jobs:
        pixels = j.scene.width * j.scene.height
        j.prepared = _StubPrepared(j.scene, pixels * min(j.scene.spp, 64))
        j.tuning = {"capacity": j.prepared.capacity, "trace_shape": 2}
    before = sum(batch._working_set(j) for j in jobs)
    budget = before // 3
    r = batch.JobRunner(reserve_bytes=0)
    monkeypatch.setattr(batch, "_free_device_bytes", lambda: budget)
    r.fit_capacities(jobs)
    after = sum(batch._working_set(j) for j in jobs)
    assert after <= budget < before
    for j in jobs:
        pixels = j.scene.width * j.scene.height
        assert j.prepared.capacity % pixels == 0 and j.prepared.capacity >= pixels
        assert j.tuning["trace_shape"] == 2
    # Working memory the autotuner's probes already hold is not needed again.
    j0 = max(jobs, key=batch._working_set)
    need = batch._working_set(j0)
    j0.held_bytes = need // 2
    assert batch._working_set(j0) == need - need // 2
    j0.held_bytes = 10 * need
    assert batch._working_set(j0) == 0
    j0.held_bytes = 0
    # A budget below one pass of every job leaves each job at one pass.
    monkeypatch.setattr(batch, "_free_device_bytes", lambda: 1)
    r.fit_capacities(jobs)
    assert all(j.prepared.capacity == j.scene.width * j.scene.height for j in jobs)
