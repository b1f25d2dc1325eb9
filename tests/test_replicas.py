"""Multi-process bookkeeping of `bench.py --gpus N` (replicas, no exchange
step), run as two gloo ranks on the CPU: every rank sees the slowest rank's
time, the value counts the rays of all ranks, and the ranks trace different
ray sets."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, ws, port, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    from yaoray_b200 import scenes

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        mine = 10.0 * (rank + 1)
        slowest = bench.max_over_ranks(mine, ws, "cpu")
        rays = scenes.incoherent_rays(1000, seed=bench.replica_ray_seed(rank))
        out.put((rank, slowest, bench.replica_value(ws, 1000, 3, slowest), rays[:4].copy()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_reduce_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, v0, rays0), (r1, s1, v1, rays1) = got
    assert (r0, r1) == (0, 1)
    assert s0 == s1 == 20.0
    assert v0 == v1 == 2 * 1000 * 3 / 0.020 / 1e6
    assert not np.array_equal(rays0, rays1)
