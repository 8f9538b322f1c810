"""bench.py's multi-GPU plumbing (replicas only) with world_size 2 over gloo
on CPU: the timed region's max over ranks and the whole-job throughput."""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    r, w, local = bench.dist_setup(world)
    ms = 100.0 + 50.0 * r                     # rank 1 is the slow one
    bench.barrier()
    m = bench.max_over_ranks(ms)
    v = bench.whole_job_value(1000.0, w, m)
    q.put((r, w, m, v))
    import torch.distributed as dist
    dist.destroy_process_group()


def test_two_rank_aggregation():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, w, m, v in out:
        assert w == 2 and m == 150.0
        assert v == pytest.approx(2 * 1000.0 / 0.150)
