"""Replica bookkeeping of bench.py under torch.distributed, on CPU with gloo (world size 2).

The step does not shard across GPUs: each rank steps its own replica and the only
exchange is the timing/throughput reduction (max of the per-rank time, sum of the
particles). This runs that reduction with two CPU ranks.
"""
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update({"MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "RANK": str(rank),
                       "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank)})
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    w, r, lr = bench.dist_env()
    t = bench.max_over_ranks(10.0 + rank, w)
    p = bench.sum_over_ranks(1000.0 * (rank + 1), w)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, w, r, lr, t, p))


def test_replica_reductions_two_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, w, r, lr, t, p in res:
        assert (w, r, lr) == (2, rank, rank)
        assert t == 11.0          # max over ranks of the timed region
        assert p == 3000.0        # particles of all replicas


def test_single_rank_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.sum_over_ranks(7.0, 1) == 7.0


@pytest.mark.parametrize("scale", [1.0, 0.5])
def test_benchmark_scene_sizes(mf, scale):
    """The benchmark scene: 714 x 214 workpiece lattice plus the sampled tool."""
    sys.path.insert(0, str(ROOT))
    import bench

    p = bench.cut_params(mf, nx=int(round(714 * scale)), ny=int(round(214 * scale)), dx=2.8e-4 / scale)
    sc = mf.Scene.from_params(p)
    assert sc.s.n_workpiece == int(round(714 * scale)) * int(round(214 * scale))
    assert sc.s.n_tool > 0 and sc.N == sc.s.n_workpiece + sc.s.n_tool
    if scale == 1.0:
        assert sc.N == 176695
