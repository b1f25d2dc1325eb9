#!/usr/bin/env python3
"""Traversal benchmark: Mrays/s of incoherent closest-hit rays on the
2,097,152-triangle traversal set (512 noisy spheres x 4096 triangles in a 100^3
box; 7,997,584 rays per step, origins uniform in the box, directions uniform).

One step = one closest-hit trace of all 7,997,584 rays through the reference's
SAH BVH (same layout as BuildBvh). Inputs (256 MB of rays, 128 MB of hits,
~150 MB of BVH) exceed the 126 MB L2, so no L2 flush is needed between steps.

  value      device throughput: rays resident in HBM, K launches timed with
             CUDA events on the launching stream (max over ranks).
  e2e        the same metric through the C ABI's host entry point
             (yrc_trace_host): pinned host rays in, host hits out, the copies
             inside the timed region.
  roofline   algorithmic bytes per launch = sum over rays of
             32 * node_tests + 48 * triangle_tests + 32 (ray) + 16 (hit),
             with the reference's own BvhTraceStats counts, / kernel time,
             against the measured HBM copy bandwidth.
  cpu_baseline  the reference CPU traversal (IntersectBvh, compiled from the
             reference sources) on this host's cores, on a bounded sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU (weak scaling, replicas: each rank traces its own ray set):
  python -m torch.distributed.run --nproc-per-node N bench.py --gpus N ...
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mrays/s traversal"
UNIT = "Mrays/s"
WORKLOAD = "traversal-2M-tris-incoherent-closest-hit"
RAYS_PER_STEP = 2828 * 2828
PROFILE_SUMMARY = ROOT / "profiles" / "trace_closest_incoherent_2M.md"


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# Replicas (one process per GPU, no exchange step): each rank traces its own
# ray set; the job's time is the slowest rank's device time and its value the
# rays of all ranks over that time.
def replica_ray_seed(rank: int) -> int:
    return 2 + 1000 * rank


def max_over_ranks(ms: float, ws: int, device) -> float:
    import torch
    import torch.distributed as dist

    t = torch.tensor([ms], dtype=torch.float64, device=device)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(ws: int, rays_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job Mrays/s of `ws` replicas."""
    return ws * rays_per_rank * steps / (max_ms / 1e3) / 1e6


class ClockSampler:
    """Samples the SM clock, power and throttle reasons during the timed region:
    through NVML every 10 ms where its bindings load (so that a timed region of
    tens of milliseconds still gets several samples), else through nvidia-smi
    every 0.2 s. Reads only; changes no setting of the GPU."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._handle = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._handle = self._device_handle(gpu_index)
        except Exception:
            self._nvml = None

    def _device_handle(self, idx: int):
        """The NVML handle of CUDA device idx, matched by PCI address (CUDA and
        NVML may number the visible GPUs differently)."""
        n = self._nvml
        try:
            import torch

            prop = torch.cuda.get_device_properties(idx)
            bus = f"{prop.pci_domain_id:08x}:{prop.pci_bus_id:02x}:{prop.pci_device_id:02x}.0"
            return n.nvmlDeviceGetHandleByPciBusId_v2(bus)
        except Exception:
            return n.nvmlDeviceGetHandleByIndex(idx)

    def _sample_nvml(self):
        n, h = self._nvml, self._handle
        sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
        mx = n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)
        watts = n.nvmlDeviceGetPowerUsage(h) / 1000.0
        bits = n.nvmlDeviceGetCurrentClocksEventReasons(h)
        flags = [n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                 n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap]
        return [str(sm), str(mx), f"{watts:.2f}"] + ["Active" if bits & f else "Not Active" for f in flags]

    def _run(self):
        while not self._stop.is_set():
            try:
                if self._nvml is not None:
                    self.rows.append(self._sample_nvml())
                    self._stop.wait(0.01)
                    continue
                out = subprocess.run(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                if out.returncode == 0 and out.stdout.strip():
                    self.rows.append([c.strip() for c in out.stdout.strip().split(",")])
            except Exception:
                self._nvml = None  # fall back to nvidia-smi
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._thread:
            self._thread.join(timeout=10)
        if self._nvml is not None:
            try:
                self._nvml.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows),
                "source": "nvml" if self._handle is not None and self._nvml is not None else "nvidia-smi"}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profiled_traffic(rays: int):
    """DRAM bytes (read + write) of one trace launch over `rays` rays: the
    per-ray figure of the committed ncu capture (a 1M-ray launch of the same
    workload) scaled by the ray count."""
    if PROFILE_SUMMARY.exists():
        m = re.search(r"dram_bytes_per_ray:\s*([0-9.eE+]+)", PROFILE_SUMMARY.read_text())
        if m:
            return round(float(m.group(1)) * rays)
    return None


def cpu_baseline(geom, rays, seconds: float = 10.0):
    """Times the reference CPU traversal (oracle/_ref, else the C oracle port)
    on all host threads over repeated 1M-ray chunks for ~`seconds`."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    threads = os.cpu_count() or 1
    chunk = rays[: 1 << 20]
    if oracle.ref_available():
        scene = oracle.RefScene(geom, threads=threads)
        run = lambda: scene.trace_count(chunk, any_hit=False, threads=threads)  # noqa: E731
        kind = "reference"
    else:
        from yaoray_b200 import accel
        scene = oracle.OracleScene(geom, accel.build_bvh(geom))
        run = lambda: scene.trace(chunk, threads=threads, stats=False)  # noqa: E731
        kind = "port"
    run()  # warm-up
    done = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        run()
        done += chunk.shape[0]
    dt = time.perf_counter() - t0
    return {"value": done / dt / 1e6, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"{done} incoherent closest-hit rays ({done // chunk.shape[0]} x 1M-ray chunks of the same "
                      f"workload) in {dt:.1f} s on {threads} threads"}


def run_reference(args):
    """--impl reference: the reference's own CPU IntersectBvh on all host
    threads over the same 7,997,584 incoherent rays per step as the GPU arm
    (same scene, BVH builder, ray seed and count)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    from yaoray_b200 import scenes
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    geom = scenes.traversal_scene()
    rays = scenes.incoherent_rays(args.rays, seed=replica_ray_seed(0))
    n = rays.shape[0]
    threads = os.cpu_count() or 1
    if oracle.ref_available():
        scene = oracle.RefScene(geom, threads=threads)
        kind = "reference"
        step = lambda: scene.trace_count(rays, False, threads)  # noqa: E731
    else:
        from yaoray_b200 import accel
        scene = oracle.OracleScene(geom, accel.build_bvh(geom))
        kind = "port"
        step = lambda: scene.trace(rays, threads=threads, stats=False)  # noqa: E731
    for _ in range(args.warmup):
        step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step()
    dt = time.perf_counter() - t0
    value = args.steps * n / dt / 1e6
    line = {"metric": METRIC, "value": round(value, 3), "unit": UNIT, "impl": "reference", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt / args.steps * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "triangles": geom.triangle_count, "rays_per_step": n,
                       "ray_set": "incoherent: origin U[0,100]^3, direction uniform", "threads": threads},
            "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"all {n} incoherent rays of a step, {args.steps} steps"},
            "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_gpu(args):
    import torch
    import torch.distributed as dist

    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    from yaoray_b200 import accel, scenes

    geom = scenes.traversal_scene()
    t0 = time.perf_counter()
    bvh, on_device = accel.build_bvh_device(geom)  # the reference's bytes, built on the GPU
    build_device_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    host_bvh = accel.build_bvh(geom)  # the same build on the host's threads, for comparison
    build_host_s = time.perf_counter() - t0
    assert on_device and host_bvh.nodes.tobytes() == bvh.nodes.tobytes()
    del host_bvh
    acc = accel.DeviceAccelerator(geom, bvh)
    rays_np = scenes.incoherent_rays(args.rays, seed=replica_ray_seed(rank))
    n = rays_np.shape[0]
    rays = torch.from_numpy(rays_np).to(dev)
    hits = torch.empty((n, 4), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    # Algorithmic bytes per launch from the per-ray BvhTraceStats counts.
    with torch.cuda.stream(stream):
        st = acc.trace_stats(rays, stream=stream)
    stream.synchronize()
    node_tests = int(st[0].to(torch.int64).sum().item())
    tri_tests = int(st[1].to(torch.int64).sum().item())
    algo_bytes = 32 * node_tests + 48 * tri_tests + (32 + 16) * n
    del st
    # Device BVH: one 32-byte box+ref per node (stored as 64-byte child pairs)
    # and one 48-byte record per triangle.
    bvh_mib = (32 * len(bvh.nodes) + 48 * geom.triangle_count) >> 20

    def barrier():
        if ws > 1:
            dist.barrier()

    # Autotuner: pick the fastest compiled launch shape on a 2M-ray slice of
    # this step's rays (untimed).
    if args.four_wide:  # opt-in four-wide traversal of the same BVH (same hits)
        acc.set_wide(True)
    if args.ray_order != "off":  # opt-in ray reordering before each trace (same hits)
        acc.set_ray_order(args.ray_order, 19, 0.05)
    if args.trace_shape is not None:  # a shape fixed by the caller (e.g. to profile the one a plain run chose)
        acc.set_trace_shape(args.trace_shape)
        tune = {"shape": args.trace_shape, "times_ms": None}
    else:
        tune = acc.autotune(rays[: min(n, 1 << 21)], stream=stream)

    for _ in range(args.warmup):
        acc.intersect(rays, hits=hits, stream=stream)
    stream.synchronize()
    acc.check()

    gpu_index = int(os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local]) \
        if os.environ.get("CUDA_VISIBLE_DEVICES") else local
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(gpu_index) as clocks:
        start.record(stream)
        for _ in range(args.steps):
            acc.intersect(rays, hits=hits, stream=stream)
        end.record(stream)
        end.synchronize()
    torch.cuda.synchronize()
    barrier()
    elapsed_ms = start.elapsed_time(end)
    acc.check()
    max_ms = max_over_ranks(elapsed_ms, ws, dev)
    per_launch_s = elapsed_ms / 1e3 / args.steps
    value = replica_value(ws, n, args.steps, max_ms)

    # End to end through the C ABI host path (pinned host buffers).
    host_rays = torch.from_numpy(rays_np).pin_memory().numpy()
    host_hits = torch.empty((n, 4), dtype=torch.float32).pin_memory().numpy()
    # The host path's own launch shape (its kernels share the GPU with its
    # copies), tuned untimed on a 2M-ray slice of the step's host rays.
    host_tune = {"shape": args.trace_shape} if args.trace_shape is not None else \
        acc.autotune_host(host_rays[: min(n, 1 << 21)])
    if args.trace_shape is not None:
        acc.set_host_trace_shape(args.trace_shape)
    for _ in range(max(1, args.warmup // 2)):
        acc.intersect_host(host_rays, out=host_hits)
    e_steps = max(1, args.steps // 2)
    barrier()
    t0 = time.perf_counter()
    for _ in range(e_steps):
        acc.intersect_host(host_rays, out=host_hits)
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3, ws, dev)
    e2e_value = replica_value(ws, n, e_steps, e2e_ms)

    # The workload's other two query sets, timed the same way (device-resident,
    # CUDA events, max over ranks): coherent primary rays (closest hit) and
    # shadow queries (any hit, t_max = distance to a uniform random point).
    del host_rays, host_hits
    other_sets = {}
    for key, make, any_hit in (("coherent_closest_hit", lambda: scenes.coherent_rays(), False),
                               ("incoherent_any_hit_shadow", lambda: scenes.shadow_rays(seed=1 + replica_ray_seed(rank)), True)):
        set_rays = torch.from_numpy(make()).to(dev)
        m = set_rays.shape[0]
        if any_hit:
            out = torch.empty(m, dtype=torch.uint8, device=dev)
        else:
            out = hits[:m] if m <= n else torch.empty((m, 4), dtype=torch.float32, device=dev)
        acc.autotune(set_rays[: min(m, 1 << 21)], any_hit=any_hit, stream=stream)
        for _ in range(args.warmup):
            acc.intersect(set_rays, any_hit=any_hit, hits=None if any_hit else out,
                          occluded=out if any_hit else None, stream=stream)
        barrier()
        torch.cuda.synchronize()
        start.record(stream)
        for _ in range(args.steps):
            acc.intersect(set_rays, any_hit=any_hit, hits=None if any_hit else out,
                          occluded=out if any_hit else None, stream=stream)
        end.record(stream)
        end.synchronize()
        acc.check()
        set_ms = max_over_ranks(start.elapsed_time(end), ws, dev)
        other_sets[key] = {"rays_per_step_per_gpu": m,
                           "mrays_s": round(replica_value(ws, m, args.steps, set_ms), 2)}
        del set_rays, out

    peak, peak_kind = measured_peak()
    achieved = algo_bytes / per_launch_s / 1e9
    traffic = profiled_traffic(n)
    base = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        base = cpu_baseline(geom, rays_np, seconds=args.cpu_seconds)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(max_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "triangles": geom.triangle_count, "bvh_nodes": int(len(bvh.nodes)),
                       "rays_per_step_per_gpu": n, "ray_set": "incoherent: origin U[0,100]^3, direction uniform",
                       "l2": f"inputs larger than L2 (rays {n * 32 >> 20} MiB + hits {n * 16 >> 20} MiB + "
                             f"BVH {bvh_mib} MiB, L2 126 MB), no flush",
                       "parallelism": f"replicas x{ws}", "launch_shape": tune["shape"],
                       "host_path_launch_shape": host_tune["shape"], "host_path_autotune_ms": host_tune.get("times_ms"),
                       "hierarchy": "four-wide copy of the reference BVH" if acc.wide else "binary reference BVH",
                       "autotune_ms": tune["times_ms"],
                       "bvh_build_s": {"device": round(build_device_s, 3), "host": round(build_host_s, 3),
                                       "host_threads": os.cpu_count()}},
            "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": n * 32,
                    "d2h_bytes_per_step": n * 16},
            "gpu_launches": args.steps,
            "roofline": {"bound": "latency", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "peak_source": f"{peak_kind} hbm_gbs",
                         "bound_note": "dependent node fetches served mostly by L1/L2, and lane divergence "
                                       "(ncu: lanes active per instruction, long-scoreboard stalls); achieved/frac "
                                       "count the algorithmic bytes against HBM, dram_frac the DRAM bytes "
                                       "the kernel really moves",
                         "dram_achieved": round(traffic / per_launch_s / 1e9, 1) if traffic else None,
                         "dram_frac": round(traffic / per_launch_s / 1e9 / peak, 4) if traffic else None,
                         "algorithmic_bytes_per_launch": algo_bytes,
                         "node_tests_per_ray": round(node_tests / n, 2),
                         "triangle_tests_per_ray": round(tri_tests / n, 2)},
            "other_ray_sets": other_sets,
            "cpu_baseline": base,
            "clocks": clocks.summary(),
        }
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return line if rank == 0 else None


# The other halves of the metric, run after the traversal line at N = 1 as
# their own processes (their own memory, device-timed regions, CPU baselines
# and clock samples): the Cornell box at its configured size, the instanced
# scene, and the radiance cache's equal-relMSE ratio.
EXTRA_LEGS = (("cornell", ["--workload", "cornell", "--steps", "10", "--warmup", "3"]),
              ("instanced", ["--workload", "instanced", "--steps", "4", "--warmup", "3"]),
              ("nrc", ["--workload", "nrc"]),
              ("jobs", ["--workload", "jobs", "--schedules", "one_at_a_time,shared,pooled"]))


def run_extra_legs():
    legs = {}
    for name, argv in EXTRA_LEGS:
        t0 = time.perf_counter()
        res = subprocess.run([sys.executable, str(ROOT / "bench.py"), *argv], capture_output=True, text=True,
                             timeout=1200)
        leg = None
        for row in reversed(res.stdout.splitlines()):
            if row.startswith("{"):
                leg = json.loads(row)
                break
        if leg is None:
            leg = {"error": f"exit {res.returncode}: {res.stderr.strip()[-600:]}"}
        leg["leg_wall_s"] = round(time.perf_counter() - t0, 1)
        legs[name] = leg
    return legs


RENDER_WORKLOADS = {
    "cornell": ("samples/s (plain MIS path tracer, Cornell box)", "cornell-256x256-64spp-depth8"),
    "instanced": ("samples/s (plain wavefront path tracer, instanced scene)",
                  "instanced-256inst-31M-tris-1920x1080-depth16"),
    "textured": ("samples/s (MIS path tracer, textured Cornell box)", "cornell-textured-256x256-64spp-depth8"),
    "cutout": ("samples/s (MIS path tracer, Cornell box with alpha cut-outs)", "cornell-cutout-256x256-64spp-depth8"),
}


def render_scene(workload: str, spp: int, size=None, max_depth=None):
    """The workload's scene; `size` (W, H) and `max_depth` override the
    configured ones (smaller cases for profiler captures only)."""
    kw = {}
    if size:
        kw.update(width=size[0], height=size[1])
    if max_depth:
        kw.update(max_depth=max_depth)
    if workload in ("cornell", "textured", "cutout"):
        from yaoray_b200 import cornell
        return {"cornell": cornell.scene, "textured": cornell.textured_scene,
                "cutout": cornell.cutout_scene}[workload](**kw)
    from yaoray_b200 import instanced
    return instanced.scene(spp=spp, **kw)


def run_render(args):
    """--workload cornell: the plain MIS path tracer on the Cornell box
    (256x256, 64 spp, Owen-Sobol seed 0, max depth 8); one step = one full
    64-spp render. --workload textured / cutout: the same box with
    reflectance textures under every filter and a normal map, and with alpha
    cut-outs and textured thin glass on top of that.
    --workload instanced: the instanced scene (256 affine instances of four
    procedural meshes, 31.4M instanced triangles, HDRI + 64 emissive
    triangles, 1920x1080, max depth 16); one step = one render of
    --render-spp samples per pixel (the full 256 spp is 256/--render-spp
    steps).
    Both go through CudaBackend.render (device-resident scene, film read back
    to the host); value = samples/s from the device time of the render,
    e2e from the host wall clock around the call. The CPU baseline renders the
    same scene with the reference CPU backend on all host threads at a few spp."""
    import torch
    from yaoray_b200.render import CudaBackend, pinned_film

    size = tuple(int(v) for v in args.size.split("x")) if args.size else None
    scene = render_scene(args.workload, args.render_spp, size, args.max_depth)
    backend = CudaBackend()
    t0 = time.perf_counter()
    prepared = backend.prepare(scene)
    prepare_s = time.perf_counter() - t0
    cache = None
    if args.cache:  # radiance cache attached (profiler captures of its kernels)
        from yaoray_b200.nrc import RadianceCache
        lo = scene.geometry.positions.min(0)
        cache = RadianceCache(lo, float((scene.geometry.positions.max(0) - lo).max()), seed=1)
        prepared.set_radiance_cache(cache, spread_threshold=1.0e-4, train_steps=2, averaged=True)
    tuning = None
    if args.tuning:  # capacity,shape fixed by the caller (e.g. to profile what a plain run chose)
        cap, shape = (int(x) for x in args.tuning.split(","))
        tuning = {"capacity": cap, "trace_shape": shape, "fixed": True}
        prepared.set_tuning(tuning)
    elif not args.no_autotune:
        t0 = time.perf_counter()
        tuning = prepared.autotune()
        tuning["seconds"] = round(time.perf_counter() - t0, 2)
    for _ in range(args.warmup):
        res = backend.render(prepared)
        assert res.ok, res.error
    gpu_index = 0
    times, devs, launches = [], [], 0
    film_buf = pinned_film(scene.width, scene.height)  # the caller's pinned film, kept across steps
    with ClockSampler(gpu_index) as clocks:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            res = backend.render(prepared, film_out=film_buf)
            times.append(time.perf_counter() - t0)
            devs.append(res.stats["device_seconds"])
            launches += int(res.stats["kernel_launches"])
    samples = scene.width * scene.height * scene.spp
    dt = sum(times) / len(times)
    ddt = sum(devs) / len(devs)
    base = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        if oracle.ref_available():
            job = oracle.RefJob.from_scene(scene)
            job.render(spp=1)
            base_spp = 4 if args.workload == "instanced" else 64  # the full Cornell jobs; 4 spp of the instanced one
            film, st, secs = job.render(spp=base_spp)
            base = {"value": round(scene.width * scene.height * base_spp / secs, 1), "unit": "samples/s",
                    "cores": os.cpu_count(), "kind": "reference",
                    "sample": f"reference CpuBackend, same scene at {base_spp} spp ({secs:.2f} s)"}
    metric, workload = RENDER_WORKLOADS[args.workload]
    config = {"workload": workload + (" (size/depth override)" if args.size or args.max_depth else "")
                          + (" (radiance cache attached)" if args.cache else ""),
              "triangles": scene.geometry.triangle_count,
              "width": scene.width, "height": scene.height, "spp_per_step": scene.spp,
              "max_depth": scene.max_depth,
              "path_segments_per_step": int(res.stats["rays_traced"]),
              "shadow_rays_per_step": int(res.stats["shadow_rays"]),
              "queue_capacity": prepared.capacity, "autotune": tuning}
    if args.workload == "instanced":
        from yaoray_b200 import instanced
        config.update(instances=int(instanced.INSTANCES), instanced_triangles=instanced.instanced_triangles(scene),
                      hdri="2048x1024 RGBA32F", emissive_triangles=int(scene.emissive.size),
                      prepare_seconds=round(prepare_s, 2))
    line = {"metric": metric, "value": round(samples / ddt, 1),
            "unit": "samples/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ddt * 1e3, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic", "config": config,
            "e2e": {"value": round(samples / dt, 1), "unit": "samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": scene.width * scene.height * 56},
            "path_segments_per_s": round(res.stats["rays_traced"] / ddt, 1),
            "shadow_rays_per_s": round(res.stats["shadow_rays"] / ddt, 1),
            "gpu_launches": launches,
            "cpu_baseline": base, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def run_nrc(args):
    """--workload nrc: equal-relMSE time of the neural-cached path tracer
    against the plain one on the instanced scene (max depth 16, radiance
    clamp 20 for every render so that the reference integrator's rare
    numerically extreme samples do not dominate the error), per frame of a
    seeded camera orbit, in steady state.

    The cached tracer renders a 60-frame orbit (0.5 degrees per frame about
    the vertical axis, a new sampler seed per frame) at --nrc-spp samples per
    pixel, training the cache online in every frame (--nrc-train-steps
    optimiser steps per batch on that frame's own unbiased training paths)
    and querying the moving average of its parameters. Nothing is trained
    outside the frames themselves, and every frame is charged its own
    training. The scene stays resident, as in an interactive renderer: each
    frame is a view update (yrc_render_scene_set_view) and one render call,
    its time the device time of the render and, beside it, the host wall
    clock around the call (film read back included). The last
    --nrc-eval-frames frames are evaluated: per frame a reference of
    --ref-spp samples per pixel of the plain tracer accumulated in FP64 over
    renders of other seeds, and the plain tracer's curve of time against
    relMSE (resident scenes of 1..64 spp, each rendered once untimed before,
    then a view update and a timed render per evaluated frame). For each
    evaluated frame the time the plain tracer needs for the cached frame's
    relMSE is interpolated on that curve; value = the geometric mean over the
    evaluated frames of that device time / the cached frame's device time,
    wall_time_ratio the same with wall times."""
    import dataclasses

    import torch
    from yaoray_b200 import instanced
    from yaoray_b200.nrc import RadianceCache
    from yaoray_b200.render import CudaBackend, build_two_level_bvh, pinned_film

    W, H, CLAMP, C_SPREAD, DECAY, ORBIT_DEG = args.nrc_width, args.nrc_height, 20.0, 1.0e-4, 0.995, 0.5
    FRAMES, EVAL, SPP = args.nrc_frames, args.nrc_eval_frames, args.nrc_spp
    base = instanced.scene(width=W, height=H, spp=1)
    base.radiance_clamp = CLAMP
    accel = build_two_level_bvh(base.geometry)

    def view(k):  # orbit frame k; the last frame is the canonical view
        return instanced.camera(orbit=math.radians((k - FRAMES + 1) * ORBIT_DEG))

    def scene(spp, seed, k):
        return dataclasses.replace(base, spp=spp, seed=seed, camera=view(k))

    def relmse(img, ref):
        return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))

    backend = CudaBackend()
    lo = base.geometry.positions.min(0)
    extent = float((base.geometry.positions.max(0) - lo).max())

    # The render autotuner's queue capacity and launch shape per spp level,
    # found on the plain tracer at the canonical view and used by both tracers.
    levels = (1, 2, 4, 8, 16, 32, 64)
    tunings = {}
    if not args.no_autotune:
        for spp in sorted(set(levels) | {SPP}):
            p = backend.prepare(scene(spp, 7, FRAMES - 1), accel)
            tunings[spp] = p.autotune()
            p.close()

    def prepare(spp, seed, k):
        p = backend.prepare(scene(spp, seed, k), accel)
        if spp in tunings:
            p.set_tuning(tunings[spp])
        return p

    # One pinned film buffer for every timed frame, as an interactive
    # renderer keeps its framebuffer (the image is taken from it before the
    # next render).
    film_buf = pinned_film(W, H)

    def timed_render(p):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = backend.render(p, film_out=film_buf)
        wall = time.perf_counter() - t0
        return r.linear(), r.stats, wall

    evaluated = list(range(FRAMES - EVAL, FRAMES))
    refs, curves = {}, {k: [] for k in evaluated}
    for k in evaluated:
        ref = np.zeros((H, W, 3), np.float64)
        per = min(128, args.ref_spp)
        p = backend.prepare(scene(per, 1000 + 97 * k, k), accel)
        for j in range(max(1, args.ref_spp // per)):
            p.set_view(view(k), 1000 + 97 * k + j)
            ref += backend.render(p).linear()
        p.close()
        refs[k] = ref / max(1, args.ref_spp // per)
    for spp in levels:
        p = prepare(spp, 1, 0)
        backend.render(p)  # allocation and capture, untimed
        for k in evaluated:
            p.set_view(view(k), 5000 + 13 * k + spp)
            img, st, wall = timed_render(p)
            curves[k].append((spp, relmse(img, refs[k]), st["device_seconds"], wall))
        p.close()

    cache = RadianceCache(lo, extent, seed=1)
    cache.set_average_decay(DECAY)
    frames = []
    launches = 0
    p = prepare(SPP, 100, 0)
    p.set_radiance_cache(cache, spread_threshold=C_SPREAD, train_steps=args.nrc_train_steps, averaged=True)
    with ClockSampler(0) as clocks:
        for k in range(FRAMES):
            p.set_view(view(k), 100 + k)
            img, st, wall = timed_render(p)
            launches += int(st["kernel_launches"])
            frames.append({"frame": k, "ms": st["device_seconds"] * 1e3, "wall_ms": wall * 1e3,
                           "relmse": relmse(img, refs[k]) if k in refs else None,
                           "cache_queries": int(st["cache_queries"]), "path_segments": int(st["rays_traced"])})
    p.close()
    cache.check()
    cache.close()

    def plain_time_for(curve, err, col):
        pts = sorted(curve, key=lambda x: -x[1])  # decreasing error
        for a, b in zip(pts, pts[1:]):
            if b[1] <= err <= a[1]:
                f = (np.log(err) - np.log(a[1])) / (np.log(b[1]) - np.log(a[1]))
                return float(np.exp(np.log(a[col]) + f * (np.log(b[col]) - np.log(a[col]))))
        last = pts[-1] if err < pts[-1][1] else pts[0]
        return float(last[col] * last[1] / err)  # beyond the curve: relMSE ~ 1 / time

    per_frame = []
    for f in frames:
        k = f["frame"]
        if k not in refs:
            continue
        dev = plain_time_for(curves[k], f["relmse"], 2) / (f["ms"] / 1e3)
        wall = plain_time_for(curves[k], f["relmse"], 3) / (f["wall_ms"] / 1e3)
        per_frame.append({"frame": k, "cached_ms": round(f["ms"], 3), "cached_wall_ms": round(f["wall_ms"], 2),
                          "relmse": round(f["relmse"], 5), "cache_queries": f["cache_queries"],
                          "path_segments": f["path_segments"], "ratio_device_time": round(dev, 3),
                          "ratio_wall_time": round(wall, 3),
                          "plain": [{"spp": s_, "relmse": round(e, 5), "ms": round(t * 1e3, 3),
                                     "wall_ms": round(w_ * 1e3, 2)} for s_, e, t, w_ in curves[k]]})
    value = float(np.exp(np.mean([np.log(x["ratio_device_time"]) for x in per_frame])))
    wall_value = float(np.exp(np.mean([np.log(x["ratio_wall_time"]) for x in per_frame])))
    train_ms = [f["ms"] for f in frames]
    line = {"metric": "equal-relMSE time ratio, plain / neural-cached (instanced scene, steady-state orbit frames)",
            "value": round(value, 3), "unit": "x", "n_gpus": 1, "steps": EVAL, "warmup": FRAMES - EVAL,
            "ms_per_step": round(float(np.mean([x["cached_ms"] for x in per_frame])), 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 render, bf16 MLP", "data": "synthetic",
            "config": {"workload": f"instanced-{W}x{H}-depth16-clamp20-orbit{FRAMES}", "reference_spp": args.ref_spp,
                       "reference_accumulation": "fp64", "spread_threshold": C_SPREAD, "spp_per_frame": SPP,
                       "train_steps_per_batch": args.nrc_train_steps,
                       "orbit": f"{FRAMES} frames, {ORBIT_DEG} degrees apart about the vertical axis, a new sampler "
                                "seed per frame; the cache trains online in every frame and nowhere else",
                       "evaluated_frames": evaluated, "timing": "resident scenes, a view update and one render call "
                       "per frame (the cache's first frame includes allocation and capture); device time from "
                       "events around the render, wall time from the host clock around the call",
                       "queue_capacity_per_spp": {s_: t["capacity"] for s_, t in tunings.items()},
                       "cache": "16x2^19x2 hash grid + SH4, 64x5 MLP, bf16 tcgen05, Adam 1e-2, "
                                f"parameter moving average {DECAY}",
                       "orbit_frame_ms": {"first": round(train_ms[0], 3), "median": round(float(np.median(train_ms)), 3),
                                          "median_wall": round(float(np.median([f["wall_ms"] for f in frames])), 3)}},
            "per_frame": per_frame,
            "wall_time_ratio": round(wall_value, 3),
            "gpu_launches": launches,
            "e2e": {"value": round(wall_value, 3), "unit": "x", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": W * H * 56,
                    "note": "the same ratio from host wall clock around each render call (films read back)"},
            "cpu_baseline": None, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def run_jobs(args):
    """--workload jobs: 48 uneven render jobs (resolutions 128^2..1024^2, spp
    16..1024 scaled by --spp-scale, 10K-2M-triangle sphere-mesh scenes with
    the instanced material mix plus subsurface, half with a radiance cache),
    rendered once untimed (allocation and graph capture), then under each of
    --schedules: one at a time, concurrently from --concurrency worker
    threads (one stream per job), in shared launches (groups of
    --concurrency jobs, one graph launch per step for all unfinished jobs of
    a group; device-memory admission) and in pooled launches (the same
    groups, with one traversal launch per bounce over every job's rays and
    one shade launch per material class). value = aggregate samples/s of
    the shared-launch run (the pooled run without it); the line carries
    per-job latency p50/p99 of each."""
    import torch
    from yaoray_b200 import batch

    t0 = time.perf_counter()
    jobs = batch.job_set(48, seed=7, spp_scale=args.spp_scale)
    runner = batch.JobRunner()
    runner.prepare(jobs, autotune=not args.no_autotune)
    prepare_s = time.perf_counter() - t0
    schedules = set(args.schedules.split(","))
    runner.run_sequential(jobs)  # warm-up: allocates and captures every job's batch graph
    torch.cuda.synchronize()
    runs, lat = {}, {}  # latencies are per job and overwritten by the next schedule: keep each run's
    with ClockSampler(0) as clocks:
        if "one_at_a_time" in schedules:
            runs["one_at_a_time"] = runner.run_sequential(jobs)
            lat["one_at_a_time"] = runs["one_at_a_time"].latency_quantiles()
        if "concurrent" in schedules:
            runs["concurrent"] = runner.run_concurrent(jobs, concurrency=args.concurrency)
            lat["concurrent"] = runs["concurrent"].latency_quantiles()
        if "shared" in schedules:
            runs["shared_launch"] = runner.run_shared_launch(jobs, concurrency=args.concurrency)
            lat["shared_launch"] = runs["shared_launch"].latency_quantiles()
        runs["pooled_launch"] = runner.run_shared_launch(jobs, concurrency=args.concurrency, pooled=True)
        lat["pooled_launch"] = runs["pooled_launch"].latency_quantiles()
    pooled = runs["pooled_launch"]
    # value: the shared launch (one graph launch per step holding every job's
    # batch graph), measured 1-2 % faster than the pooled form on this job set.
    main = runs.get("shared_launch", pooled)
    failed = [j.name for j in jobs if not j.ok]
    runner.close(jobs)
    tris = [j.scene.geometry.triangle_count for j in jobs]
    film_bytes = sum(j.scene.width * j.scene.height * 56 for j in jobs)
    base = None
    if not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle
        if oracle.ref_available():
            # The plain subset (jobs without a cache), one after another at 32 spp.
            plain = [j for j in jobs if not j.use_cache][:8]
            n, secs = 0, 0.0
            for j in plain:
                film, st, dt = oracle.RefJob.from_scene(j.scene).render(spp=32)
                n += j.scene.width * j.scene.height * 32
                secs += dt
            base = {"value": round(n / secs, 1), "unit": "samples/s", "cores": os.cpu_count(), "kind": "reference",
                    "sample": f"reference CpuBackend, the first {len(plain)} jobs without a cache, 32 spp each, "
                              f"one after another ({secs:.2f} s)"}
    line = {"metric": "samples/s (48 batched uneven render jobs)", "value": round(main.samples_per_s, 1),
            "unit": "samples/s", "n_gpus": 1, "steps": 1, "warmup": 1,
            "ms_per_step": round(main.wall_s * 1e3, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "jobs48-128..1024px-16..1024spp-10K..2M-tris", "jobs": len(jobs),
                       "spp_scale": args.spp_scale, "concurrency": args.concurrency,
                       "scheduling": ("shared launch: groups of up to --concurrency jobs, one yrc_render_many call "
                                      "per group, one graph launch per step for all unfinished jobs of the group"
                                      if main is not pooled else
                                      "pooled launch: groups of up to --concurrency jobs, one yrc_render_pooled call "
                                      "per group; per bounce one persistent traversal launch over every job's extend "
                                      "rays, one shade launch per material class and one shadow launch"),
                       "triangles_min_max": [min(tris), max(tris)], "with_radiance_cache": sum(j.use_cache for j in jobs),
                       "samples_total": main.samples, "prepare_seconds": round(prepare_s, 2),
                       "autotune_seconds": round(sum(j.tune_s for j in jobs), 2),
                       "capacities": sorted({j.tuning["capacity"] for j in jobs if j.tuning}),
                       "capacity_halved_jobs": sum(1 for j in jobs if j.tuning and j.tuning.get("fitted")),
                       "admission_budget_gb": round(main.extra.get("budget_bytes", 0) / 2**30, 1),
                       "peak_concurrent_jobs": main.peak_concurrency},
            **{name: {"samples_per_s": round(r.samples_per_s, 1), "wall_s": round(r.wall_s, 3),
                      "latency_p50_s": lat[name]["p50"], "latency_p99_s": lat[name]["p99"]}
               for name, r in runs.items()},
            "failed_jobs": failed,
            "gpu_launches": sum(j.kernels for j in jobs),
            "e2e": {"value": round(main.samples_per_s, 1), "unit": "samples/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": film_bytes,
                    "note": "value is already host wall clock around the CudaBackend.render calls, films read back"},
            "cpu_baseline": base, "clocks": clocks.summary()}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--workload", choices=["traversal", "cornell", "textured", "cutout", "instanced", "nrc", "jobs"],
                    default="traversal")
    ap.add_argument("--nrc-width", type=int, default=1920)
    ap.add_argument("--nrc-height", type=int, default=1080)
    ap.add_argument("--ref-spp", type=int, default=512)
    ap.add_argument("--nrc-frames", type=int, default=60, help="--workload nrc: orbit frames")
    ap.add_argument("--nrc-eval-frames", type=int, default=2, help="--workload nrc: last frames evaluated")
    ap.add_argument("--nrc-spp", type=int, default=4, help="--workload nrc: spp per orbit frame")
    ap.add_argument("--nrc-train-steps", type=int, default=2, help="--workload nrc: optimiser steps per batch")
    ap.add_argument("--spp-scale", type=float, default=1.0, help="spp scale of --workload jobs")
    ap.add_argument("--schedules", default="one_at_a_time,concurrent,shared,pooled",
                    help="--workload jobs: the schedules to time (the default bench line's leg skips 'concurrent')")
    ap.add_argument("--concurrency", type=int, default=16,
                    help="--workload jobs: jobs per shared launch (and concurrent streams)")
    ap.add_argument("--no-autotune", action="store_true", help="render workloads: keep the default queue capacity")
    ap.add_argument("--trace-shape", type=int, default=None, help="traversal: use this launch shape, no autotune")
    ap.add_argument("--four-wide", action="store_true", help="traversal: the opt-in four-wide traversal")
    ap.add_argument("--ray-order", choices=["off", "direction", "two-point"], default="off",
                    help="traversal: the opt-in ray reordering (19-bit key) before each trace")
    ap.add_argument("--tuning", default=None, help="render workloads: 'capacity,shape' instead of the autotuner")
    ap.add_argument("--render-spp", type=int, default=16, help="spp per step of --workload instanced")
    ap.add_argument("--size", default=None, help="render workloads: WxH instead of the configured size (profiling)")
    ap.add_argument("--max-depth", type=int, default=None, help="render workloads: max depth override (profiling)")
    ap.add_argument("--cache", action="store_true", help="render workloads: attach a radiance cache (profiling)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="traversal: skip the Cornell, instanced and radiance-cache legs of the default line")
    ap.add_argument("--rays", type=int, default=RAYS_PER_STEP,
                    help="rays per step (default: the full 7,997,584; smaller only for profiling captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload in RENDER_WORKLOADS:
        run_render(args)
    elif args.workload == "nrc":
        run_nrc(args)
    elif args.workload == "jobs":
        run_jobs(args)
    else:
        line = run_gpu(args)
        if line is not None:
            if line["n_gpus"] == 1 and not args.no_extras:
                line["workloads"] = run_extra_legs()
            print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
