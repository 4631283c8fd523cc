"""Replica timing reduction on two gloo ranks (CPU): max over ranks and whole-job throughput."""
import os
import socket

import pytest
import torch.multiprocessing as mp

from frontierlabproject_b200.replicas import max_over_ranks, whole_job_rate


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 100 + 10 r ms for the step and 50 - r ms inside the passes
        total, passes = max_over_ranks([100.0 + 10 * rank, 50.0 - rank], dist)
        rate = whole_job_rate(2.0e12, total / 1e3, world)
        q.put((rank, total, passes, rate))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(world))
    for rank, total, passes, rate in got:
        assert total == 110.0 and passes == 50.0
        assert rate == pytest.approx(2.0e12 * 2 / 0.110)


def test_single_process_identity_and_errors():
    assert max_over_ranks([1.5, 2.5]) == [1.5, 2.5]
    assert whole_job_rate(10.0, 2.0, 1) == 5.0
    with pytest.raises(ValueError):
        whole_job_rate(1.0, 0.0, 1)
