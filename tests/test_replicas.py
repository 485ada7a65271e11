"""The multi-process path of bench runs (one process per GPU, independent
replicas): two gloo ranks on the CPU check the barrier, the max-over-ranks
timing and the whole-job rate that rank 0 reports."""
from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from fiber3d_b200 import replicas
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        assert replicas.rank_info() == (rank, world, rank)
        replicas.barrier()
        # rank r took (10 + r) ms in total and (3 - r) ms in its e2e region
        mx = replicas.max_over_ranks([10.0 + rank, 3.0 - rank])
        rate = replicas.aggregate_rate(1000.0, 5, world, mx[0])
        replicas.barrier()
        q.put((rank, mx, rate))
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, mx, rate in got:
        assert mx == [11.0, 3.0]
        assert rate == pytest.approx(1000.0 * 5 * 2 / 11e-3)


def test_single_process_is_identity():
    from fiber3d_b200 import replicas
    assert replicas.max_over_ranks([1.5, 2.0]) == [1.5, 2.0]
    replicas.barrier()
    with pytest.raises(ValueError):
        replicas.aggregate_rate(1.0, 1, 1, 0.0)
