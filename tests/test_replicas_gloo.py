"""CPU, world_size 2 over gloo: the bench's replica plumbing.

M(X) needs no collective; N GPUs run N independent replicas and the bench
reports the whole job's time as the max over ranks.  This checks that
aggregation (dist_setup / barrier / max_over_ranks from bench.py) with two
CPU processes, no GPU involved.
"""
import os
import socket
import sys

import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update({"RANK": str(rank), "WORLD_SIZE": str(world), "LOCAL_RANK": str(rank),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port), "DR_DIST_BACKEND": "gloo"})
    sys.path.insert(0, ROOT)
    import bench

    w, r, _ = bench.dist_setup()
    bench.barrier(w)
    m = bench.max_over_ranks(1.0 + r, w)
    import torch.distributed as dist

    dist.destroy_process_group()
    q.put((r, w, m))


def test_max_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(timeout=120)
    out = sorted(q.get(timeout=5) for _ in range(2))
    assert out == [(0, 2, 2.0), (1, 2, 2.0)]
