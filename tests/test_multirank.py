"""
The multi-GPU (replica) logic on the CPU: two gloo ranks, each with its own timed region, agree
on the slowest rank's time and the whole-job throughput, as bench.py computes them under torchrun.
"""

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from qpop_diffraction_b200 import replicas
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, lr = replicas.rank_env()
        t = replicas.slowest(1.0 + rank)            # rank 1 is the slow one
        out[rank] = (r, w, lr, t, replicas.throughput(100, t, w))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_slowest_time():
    mp = pytest.importorskip("torch.multiprocessing")
    ctx = mp.get_context("spawn")
    port = _free_port()
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][:3] == (0, 2, 0) and res[1][:3] == (1, 2, 1)
    assert res[0][3] == res[1][3] == 2.0
    assert res[0][4] == res[1][4] == 100.0


def test_single_process_needs_no_group():
    from qpop_diffraction_b200 import replicas
    assert replicas.slowest(0.5) == 0.5
    assert replicas.throughput(10, 2.0, 1) == 5.0
