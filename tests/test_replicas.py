"""Replicas across ranks (host logic, CPU): the instance assignment and the
merge of per-rank results, with world size 2 over gloo."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from bdc_b200 import replicas

MIX = [(n, k) for n, k in [(16, 8), (18, 6), (20, 10), (22, 11), (24, 8), (24, 12)] for _ in range(8)]


def test_partition_is_disjoint_complete_and_balanced():
    for world in (1, 2, 3, 4, 8):
        parts = replicas.partition(MIX, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(MIX)))
        loads = [sum(replicas.instance_cost(*MIX[i]) for i in p) for p in parts]
        biggest = max(replicas.instance_cost(*x) for x in MIX)
        assert max(loads) - min(loads) <= biggest
        assert parts == replicas.partition(MIX, world)  # deterministic


def test_merge_rejects_duplicates_and_gaps():
    assert replicas.merge([[(1, {"a": 1})], [(0, {"a": 0})]], 2) == [{"a": 0}, {"a": 1}]
    with pytest.raises(ValueError):
        replicas.merge([[(0, {})], [(0, {})]], 1)
    with pytest.raises(ValueError):
        replicas.merge([[(0, {})]], 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = replicas.partition(MIX, world)[rank]
        # stand-in results: what a rank's batch would report per instance
        local = [(i, {"n": MIX[i][0], "k": MIX[i][1], "rank": rank}) for i in mine]
        merged = replicas.gather(local, len(MIX))
        if rank == 0:
            q.put(merged)
        else:
            assert merged is None
    finally:
        dist.destroy_process_group()


def test_gather_over_gloo_world_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert [(m["n"], m["k"]) for m in merged] == MIX
    assert {m["rank"] for m in merged} == {0, 1}
