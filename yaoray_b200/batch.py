"""Batched uneven render jobs: many independent scenes rendered concurrently
on one GPU.

Each job is a prepared scene (its own BVH, materials, film and CUDA stream,
`render.PreparedScene`); a pool of host worker threads renders up to
`concurrency` jobs at a time, so their batch graphs overlap on the GPU, and a
job is admitted only while its device working set fits under the admission
budget (free device memory minus a reserve). The ctypes calls release the
interpreter lock, so the workers truly overlap.

`job_set()` generates the batched-jobs workload: resolutions from {128^2,
256^2, 512^2, 1024^2}, samples per pixel from {16, 64, 256, 1024} (scaled by
`spp_scale` for bounded runs), scenes from the traversal-set generator (noisy
sphere meshes of 4096 triangles, 10K-2M triangles per scene) with the
instanced configuration's material mix plus a subsurface material
(separable tabulated BSSRDF, sigma_a U[0.01, 0.5], sigma_s U[0.5, 2] per
scene unit (mm), eta 1.33), lit by a small procedural sky; half of the jobs
attach a radiance cache.

The reference renders one job per process call; it has no batching of its
own — this module is an addition of this backend.
"""
from __future__ import annotations

import math
import threading
import time
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import instanced, scenes
from .accel import SceneGeometry
from .render import (COATED_DIFFUSE, CONDUCTOR, DIELECTRIC, DIFFUSE, OWEN_SOBOL, SUBSURFACE, CudaBackend,
                     EnvironmentMap, RenderScene, build_bssrdf_table, default_material)

RESOLUTIONS = (128, 256, 512, 1024)
SPPS = (16, 64, 256, 1024)


@dataclass
class Job:
    name: str
    scene: RenderScene
    use_cache: bool
    prepared: object = None
    cache: object = None
    prepare_s: float = 0.0
    tuning: dict | None = None
    tune_s: float = 0.0
    resident: bool = False  # rendered once: its working memory stays allocated
    held_bytes: int = 0  # working memory its autotuner probes left allocated (already on the device)
    kernels: int = 0  # device kernels the last render launched
    latency_s: float = 0.0
    device_s: float = 0.0
    samples: int = 0
    ok: bool = False
    error: str = ""
    film: object = None


def _camera(box: float, rng: np.random.Generator) -> dict:
    az = rng.uniform(0, 2 * math.pi)
    eye = np.array([box / 2 + 1.6 * box * math.cos(az), box * 0.9, box / 2 + 1.6 * box * math.sin(az)], np.float32)
    look = np.array([box / 2, box * 0.35, box / 2], np.float32)
    fwd = look - eye
    fwd = fwd / np.float32(np.sqrt(np.float32(np.dot(fwd, fwd))))
    right = np.cross(fwd, np.array([0, 1, 0], np.float32)).astype(np.float32)
    right = right / np.float32(np.sqrt(np.float32(np.dot(right, right))))
    up = np.cross(right, fwd).astype(np.float32)
    return {"origin": tuple(map(float, eye)), "forward": tuple(map(float, fwd)), "right": tuple(map(float, right)),
            "up": tuple(map(float, up)), "fov_y_radians": float(np.float32(45.0) * np.float32(math.pi) / np.float32(180))}


def job_scene(width: int, spp: int, spheres: int, seed: int, max_depth: int = 8) -> RenderScene:
    """One batched-jobs scene: `spheres` noisy sphere meshes (4096 triangles
    each) in a 100-unit box, one material per sphere from the instanced mix
    plus subsurface, a 256 x 128 procedural sky."""
    rng = np.random.default_rng(seed)
    geom = scenes.traversal_scene(seed=seed, spheres=spheres)
    pal = list(instanced.materials(rng))
    for _ in range(4):
        pal.append(default_material(kind=SUBSURFACE, sigma_a=rng.uniform(0.01, 0.5, 3).astype(np.float32),
                                    sigma_s=rng.uniform(0.5, 2.0, 3).astype(np.float32), bssrdf_eta=1.33,
                                    bssrdf_index=0))
    mats = np.stack(pal)
    prims = geom.primitives
    prims["material_index"] = rng.integers(0, len(mats), prims.size)
    normals = None
    env = EnvironmentMap(active=True, radiance=(1.0, 1.0, 1.0), strength=1.0, rotation=0.0,
                         texels=instanced.hdri(256, 128))
    env.build_distribution()
    height = width
    s = RenderScene(SceneGeometry(geom.positions, geom.indices, prims), mats, _camera(100.0, rng), width, height,
                    spp=spp, max_depth=max_depth, seed=seed, sampler=OWEN_SOBOL, normals=normals, environment=env)
    s.radiance_clamp = 20.0
    s.bssrdf_tables = [build_bssrdf_table(1.33)]
    return s


def job_set(count: int = 48, seed: int = 7, spp_scale: float = 1.0, max_triangles: int = 2 << 20) -> list[Job]:
    """The batched-jobs workload (see the module docstring)."""
    rng = np.random.default_rng(seed)
    jobs = []
    for j in range(count):
        res = int(rng.choice(RESOLUTIONS))
        spp = max(1, int(round(int(rng.choice(SPPS)) * spp_scale)))
        tris = float(np.exp(rng.uniform(np.log(10_000), np.log(max_triangles))))
        spheres = max(3, int(round(tris / 4096)))
        jobs.append(Job(name=f"job{j:02d}-{res}px-{spp}spp-{spheres * 4096}tri",
                        scene=job_scene(res, spp, spheres, seed * 1000 + j), use_cache=(j % 2 == 1)))
    return jobs


def _free_device_bytes() -> int:
    import torch
    free, _ = torch.cuda.mem_get_info()
    return int(free)


def _working_set(job: Job) -> int:
    """Device bytes a job's render still has to allocate: none once it has
    rendered (its working memory stays allocated), else the path state and queues
    for its queue capacity (the prepared scene's, else max(2^21, pixels))
    at ~640 B per path for these scenes (path state 196 B, coated-vertex
    state 80 B, extend / shadow / subsurface queues and transmittance
    ~350 B), ~760 B with a cache (its query queues), plus the film and,
    with a cache, its training-path records (~100 MB; the cache's grid and
    optimiser state were allocated with the cache itself)."""
    if job.resident:
        return 0
    pixels = job.scene.width * job.scene.height
    paths = job.prepared.capacity if job.prepared is not None else max(1 << 21, pixels)
    per = 760 if job.use_cache else 640
    need = paths * per + pixels * 80 + (100 << 20 if job.use_cache else 0)
    # The working memory the autotuner's probes left allocated is on the
    # device already (free device memory does not count it); the render
    # replaces it, so only the rest is still to allocate.
    return max(0, need - job.held_bytes)


@dataclass
class BatchResult:
    jobs: list
    wall_s: float
    samples: int
    peak_concurrency: int
    extra: dict = field(default_factory=dict)

    @property
    def samples_per_s(self) -> float:
        return self.samples / self.wall_s if self.wall_s > 0 else 0.0

    def latency_quantiles(self) -> dict:
        lat = np.array([j.latency_s for j in self.jobs if j.ok])
        if lat.size == 0:
            return {"p50": None, "p99": None}
        return {"p50": float(np.quantile(lat, 0.5)), "p99": float(np.quantile(lat, 0.99))}


class JobRunner:
    """Prepares jobs and renders them one at a time or concurrently."""

    def __init__(self, reserve_bytes: int = 8 << 30, keep_films: bool = False):
        self.backend = CudaBackend()
        self.reserve = reserve_bytes
        self.keep_films = keep_films

    def prepare(self, jobs: list[Job], autotune: bool = False) -> None:
        """Builds and uploads every job's scene, attaches the radiance caches
        and, with `autotune`, runs the render autotuner (queue capacity and
        traversal launch shape, probes without the cache) once per class of
        jobs with the same pixel count and batch bound min(spp, 64); the
        other jobs of a class take its result."""
        from .nrc import RadianceCache
        tuned: dict = {}
        for job in jobs:
            t0 = time.perf_counter()
            job.prepared = self.backend.prepare(job.scene)
            base_bytes = job.prepared.device_bytes
            if autotune:
                key = (job.scene.width * job.scene.height, min(job.scene.spp, 64))
                t1 = time.perf_counter()
                if key in tuned:
                    job.tuning = tuned[key]
                    job.prepared.set_tuning(job.tuning)
                else:
                    job.tuning = tuned[key] = job.prepared.autotune()
                job.tune_s = time.perf_counter() - t1
                job.held_bytes = max(0, job.prepared.device_bytes - base_bytes)
            if job.use_cache:
                p = job.scene.geometry.positions
                lo = p.min(0)
                job.cache = RadianceCache(lo, float((p.max(0) - lo).max()) + 1e-3, seed=1)
                job.cache.set_average_decay(0.995)
                job.prepared.set_radiance_cache(job.cache, spread_threshold=1e-4, train_steps=2, averaged=True)
            job.prepare_s = time.perf_counter() - t0
        self.fit_capacities(jobs)

    def fit_capacities(self, jobs: list[Job]) -> None:
        """Every schedule here keeps a job's working memory once it has
        rendered, so all the jobs' working sets must fit the device at once:
        while their sum exceeds free device memory less the reserve, the
        largest job's queue capacity is halved (in whole passes of its
        image, never below one pass). The films do not depend on it."""
        budget = max(_free_device_bytes() - self.reserve, 0)
        while sum(_working_set(j) for j in jobs) > budget:
            cands = [j for j in jobs if not j.resident and j.prepared is not None
                     and j.prepared.capacity >= 2 * j.scene.width * j.scene.height]
            if not cands:
                break
            job = max(cands, key=_working_set)
            pixels = job.scene.width * job.scene.height
            cap = max(pixels, job.prepared.capacity // 2 // pixels * pixels)
            shape = job.tuning["trace_shape"] if job.tuning else 0
            job.prepared.set_tuning({"capacity": cap, "trace_shape": shape})
            job.tuning = dict(job.tuning or {}, capacity=cap, trace_shape=shape, fitted=True)

    def _render(self, job: Job) -> None:
        t0 = time.perf_counter()
        res = self.backend.render(job.prepared)
        job.latency_s = time.perf_counter() - t0
        job.ok, job.error = res.ok, res.error
        job.resident = job.resident or res.ok
        job.device_s = res.stats.get("device_seconds", 0.0)
        job.samples = int(res.stats.get("samples_rendered", 0))
        job.kernels = int(res.stats.get("kernel_launches", 0))
        job.film = res.film if self.keep_films else None

    def run_sequential(self, jobs: list[Job]) -> BatchResult:
        t0 = time.perf_counter()
        for job in jobs:
            self._render(job)
        wall = time.perf_counter() - t0
        return BatchResult(list(jobs), wall, sum(j.samples for j in jobs), 1)

    def run_concurrent(self, jobs: list[Job], concurrency: int = 8, budget_bytes: int | None = None) -> BatchResult:
        """Renders up to `concurrency` jobs at once, admitting a job only while
        the working memory that running jobs still have to allocate fits the
        admission budget (`budget_bytes`, by default free device memory at
        the start minus the reserve); a job larger than the whole budget runs
        alone. Jobs that rendered before hold their memory already. Jobs are
        taken largest-first so small jobs fill the gaps at the end."""
        budget = budget_bytes if budget_bytes is not None else max(_free_device_bytes() - self.reserve, 0)
        lock = threading.Condition()
        in_use = [0]
        running = [0]
        peak = [0]
        order = sorted(jobs, key=lambda j: -j.scene.width * j.scene.height * j.scene.spp)

        def work(job: Job) -> None:
            need = _working_set(job)
            with lock:
                while in_use[0] > 0 and in_use[0] + need > budget:
                    lock.wait()
                in_use[0] += need
                running[0] += 1
                peak[0] = max(peak[0], running[0])
            try:
                self._render(job)
            finally:
                with lock:
                    in_use[0] -= need
                    running[0] -= 1
                    lock.notify_all()

        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=concurrency) as pool:
            list(pool.map(work, order))
        wall = time.perf_counter() - t0
        return BatchResult(list(jobs), wall, sum(j.samples for j in jobs), peak[0], {"budget_bytes": budget})

    def run_shared_launch(self, jobs: list[Job], concurrency: int = 8, budget_bytes: int | None = None,
                          pooled: bool = False) -> BatchResult:
        """Renders the jobs in groups of up to `concurrency` (largest first,
        admitted against the budget like run_concurrent), each group with
        one yrc_render_many call: every step of a group is ONE graph launch
        holding all of its unfinished jobs. With `pooled`, yrc_render_pooled:
        per bounce one persistent traversal launch serves the extend rays of
        every job of the group and one the shadow rays. A job's latency is
        its group's call."""
        budget = budget_bytes if budget_bytes is not None else max(_free_device_bytes() - self.reserve, 0)
        order = sorted(jobs, key=lambda j: -j.scene.width * j.scene.height * j.scene.spp)
        peak = 0
        t0 = time.perf_counter()
        i = 0
        while i < len(order):
            group, used = [order[i]], _working_set(order[i])
            i += 1
            while i < len(order) and len(group) < concurrency and used + _working_set(order[i]) <= budget:
                used += _working_set(order[i])
                group.append(order[i])
                i += 1
            peak = max(peak, len(group))
            g0 = time.perf_counter()
            results = self.backend.render_many([j.prepared for j in group], pooled=pooled)
            dt = time.perf_counter() - g0
            for job, res in zip(group, results):
                job.latency_s = dt
                job.ok, job.error = res.ok, res.error
                job.resident = job.resident or res.ok
                job.device_s = res.stats.get("device_seconds", 0.0)
                job.samples = int(res.stats.get("samples_rendered", 0))
                job.kernels = int(res.stats.get("kernel_launches", 0))
                job.film = res.film if self.keep_films else None
        wall = time.perf_counter() - t0
        return BatchResult(list(jobs), wall, sum(j.samples for j in jobs), peak, {"budget_bytes": budget})

    def close(self, jobs: list[Job]) -> None:
        for job in jobs:
            if job.prepared is not None:
                job.prepared.close()
            if job.cache is not None:
                job.cache.close()
