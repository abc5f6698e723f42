"""The N>1 path of bench.py (independent replicas, max-over-ranks timing) with
two gloo ranks on the CPU.  Each rank advances its own replica of a small
problem with the CPU oracle; the replicas must agree and the job rate must be
taken over the slowest rank."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "tests"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        from oracle.oracle import Oracle
        from sac_b200 import problems

        import _util

        P = problems.random_problem((10, 8), seed=3, types=["cont", "cont", "periodic", "periodic"])
        o = _util.start(Oracle, P)
        _util.run(o, 3)
        w = o.download()
        fake_ms = 10.0 + 5.0 * rank  # the slower rank decides
        ms = bench.max_over_ranks(fake_ms, world)
        rate = bench.job_rate(P.ncells, 3, world, ms / 1e3)
        gathered = [None] * world
        dist.all_gather_object(gathered, float(np.sum(w)))
        q.put((rank, ms, rate, gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, rate, gathered in out:
        assert ms == 15.0
        assert rate == pytest.approx(2 * 80 * 3 / 0.015)
        assert gathered[0] == gathered[1]  # identical replicas
