"""The multi-GPU form of the step is replicas only: each rank runs whole cases (a replica
of the bench workload, or its share of a batch) and nothing but the timing crosses ranks.
These CPU tests run that host logic in two gloo processes."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


class FakeCase:
    def __init__(self, name, cells):
        self.name, self.cells = name, cells


CASES = [FakeCase(f"c{i}", cells) for i, cells in enumerate([7, 3, 9, 1, 4, 4, 8, 2, 6, 5, 3, 7, 2, 9, 1])]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist

    import bench
    from nonnewlbm_b200 import studies

    d = bench.Dist()
    d.init("gloo")
    mine = studies.shard_cases(CASES, rank, world, size=lambda c: c.cells)
    names = [None] * world
    dist.all_gather_object(names, [c.name for c in mine])
    # the bench's time is the maximum over ranks
    t = d.max(10.0 + rank)
    d.barrier()
    out.put((rank, names, t, sum(c.cells for c in mine)))
    d.close()


def test_two_gloo_ranks_split_a_batch_and_take_the_max_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    names = res[0][1]
    assert names == res[1][1]                     # every rank computed the same split
    flat = [n for part in names for n in part]
    assert sorted(flat) == sorted(c.name for c in CASES)  # a partition: each case once
    assert all(r[2] == 11.0 for r in res)         # max over ranks
    loads = [r[3] for r in res]
    assert abs(loads[0] - loads[1]) <= max(c.cells for c in CASES)  # balanced by size
