"""Replicas-only multi-process path on CPU (gloo, world size 2): sharding covers
every unit once, the max/sum reductions and the final gather agree across ranks."""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp

from critmc_b200 import replicas
from critmc_b200.serve import mixed_workload


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out) -> None:
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    replicas.init("gloo", timeout_s=60)
    r, w, _ = replicas.rank_env()
    reqs = replicas.shard(mixed_workload(101, 200.0, seed=5), r, w)
    replicas.barrier()
    slowest = replicas.max_over_ranks(1.0 + r)
    total = replicas.sum_over_ranks(len(reqs))
    got = replicas.gather_to_root({"rank": r, "rids": [q.rid for q in reqs]})
    if r == 0:
        out.put((slowest, total, got))
    replicas.finish()


def test_two_gloo_ranks_shard_and_reduce():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    slowest, total, got = q.get()
    assert slowest == 2.0
    assert total == 101
    rids = sorted(i for g in got for i in g["rids"])
    assert rids == list(range(101))
    assert [g["rank"] for g in got] == [0, 1]


def test_single_process_defaults():
    assert replicas.shard(range(5), 0, 1) == [0, 1, 2, 3, 4]
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.gather_to_root(7) == [7]
    if os.environ.get("WORLD_SIZE", "1") == "1":
        assert replicas.rank_env()[1] == 1
    with pytest.raises(ValueError):
        replicas.shard(range(3), 0, 0)
