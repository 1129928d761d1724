"""The N > 1 host plumbing of bench.py under two CPU processes (gloo): the replica process group comes
from the environment (MASTER_ADDR 127.0.0.1, RANK, WORLD_SIZE), every rank passes the same barriers,
and each reported device time is the maximum over ranks.  The path is replicas only: no collective
touches the solver's data."""
from __future__ import annotations

import os
import socket

import pytest

mp = pytest.importorskip("torch.multiprocessing")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import bench

    w, r, _ = bench.dist_env()
    dist = bench.init_replicas(w, "gloo", 30)
    try:
        dist.barrier()
        q.put((r, bench.max_over_ranks(dist, [1.0 + r, 10.0 - r, 5.0])))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_report_the_max_device_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    try:
        got = dict(q.get(timeout=120) for _ in procs)
        for p in procs:
            p.join(timeout=60)
            assert p.exitcode == 0
    finally:
        for p in procs:
            if p.is_alive():
                p.kill()
    assert got == {0: [2.0, 10.0, 5.0], 1: [2.0, 10.0, 5.0]}


def test_one_process_needs_no_group():
    import bench

    assert bench.init_replicas(1) is None
    assert bench.max_over_ranks(None, [3, 4.5]) == [3.0, 4.5]
