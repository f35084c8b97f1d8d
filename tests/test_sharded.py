"""BA sharded by input strings (bdc_b200.sharded): the shard ranges and the
combination of the per-rank update statistics on CPU (world size 2 over
gloo), and on the GPU two ranks of one problem against one engine (two
processes on one device, exchanging over gloo; no kernel waits on another)."""
import math
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import PKG


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges_cover_the_representatives():
    from bdc_b200 import sharded
    for R in (1056, 262656, 4196352):
        for world in (1, 2, 3, 8):
            rs = [sharded.shard_range(R, r, world) for r in range(world)]
            assert rs[0][0] == 0 and rs[-1][1] == R
            assert all(a[1] == b[0] for a, b in zip(rs, rs[1:]))
            sizes = [r1 - r0 for r0, r1 in rs]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharded.shard_range(3, 0, 4)


def test_combined_normaliser_equals_the_whole_vector():
    # per-shard (max, sum exp(v - max)) combined = the whole vector's
    from bdc_b200 import sharded
    rng = np.random.default_rng(1)
    v = rng.normal(0, 30, 1000)
    for world in (1, 2, 5):
        cuts = [len(v) * r // world for r in range(world + 1)]
        sh = [v[a:b].max() for a, b in zip(cuts, cuts[1:])]
        z = [np.exp(v[a:b] - m).sum() for (a, b), m in zip(zip(cuts, cuts[1:]), sh)]
        S, lz = sharded.combine_update(sh, z)
        assert S == v.max()
        assert abs(lz - math.log(np.exp(v - v.max()).sum())) < 1e-12
        # every shard's normalised values sum to one overall
        tot = sum(np.exp(v[a:b] - m).sum() / math.exp(sharded.shard_log_z(S, lz, m))
                  for (a, b), m in zip(zip(cuts, cuts[1:]), sh))
        assert abs(tot - 1.0) < 1e-12


def test_exchange_tensors_live_on_the_handles_gpu_under_nccl():
    # NCCL runs one process per GPU: the exchange buffers must sit on the
    # handle's device, not on torch's current device (cuda:0 by default)
    from bdc_b200 import sharded
    assert sharded.comm_device("nccl", 3) == "cuda:3"
    assert sharded.comm_device("nccl", 0) == "cuda:0"
    assert sharded.comm_device("gloo", 3) == "cpu"


def test_comm_picks_the_engine_device_for_a_mocked_nccl_group(monkeypatch):
    import torch.distributed as tdist
    from bdc_b200 import sharded
    monkeypatch.setattr(tdist, "get_rank", lambda group=None: 1)
    monkeypatch.setattr(tdist, "get_world_size", lambda group=None: 2)
    monkeypatch.setattr(tdist, "get_backend", lambda group=None: "nccl")
    comm = sharded._Comm(None, device=5)
    assert comm.device == "cuda:5" and comm.rank == 1 and comm.world == 2


def _cpu_rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bdc_b200 import sharded
        v = np.random.default_rng(7).normal(0, 20, 999)
        r0, r1 = sharded.shard_range(len(v), rank, world)
        mine = v[r0:r1]
        comm = sharded._Comm()
        S = float(comm.reduce([mine.max()], "max")[0])
        z = float(comm.reduce([sharded.z_share(np.exp(mine - mine.max()).sum(), mine.max(), S)], "sum")[0])
        if rank == 0:
            q.put((S, math.log(z), v.max(), math.log(np.exp(v - v.max()).sum())))
    finally:
        dist.destroy_process_group()


def test_update_statistics_over_gloo_world_2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_cpu_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    S, lz, S_ref, lz_ref = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert S == S_ref and abs(lz - lz_ref) < 1e-12


# ------------------------------------------------------------- on the GPU
CASES = [("fixed", 12, 6, 8, ("dirichlet", 1.0, 0), float("-inf")),
         ("stop", 10, 5, 100000, ("uniform",), 1e-3)]


def _start(n, spec):
    from bdc_b200 import dist as bdist
    return bdist.uniform_start(n) if spec[0] == "uniform" else bdist.dirichlet_start(n, spec[1], spec[2])


def _gpu_rank(rank, world, port, q):
    import sys
    sys.path.insert(0, PKG)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        import bdc_b200
        from bdc_b200 import sharded
        res = {}
        for name, n, k, iters, spec, a in CASES:
            with bdc_b200.Engine(n, k, engine="count", device=0) as E:
                E.set_p(_start(n, spec))
                st = sharded.iterate(E, iters, a)
                p = sharded.gather_p(E)
            res[name] = (st, p)
        if rank == 0:
            q.put(res)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_ranks_match_one_engine(bdc, O):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for name, n, k, iters, spec, a in CASES:
        st, p = res[name]
        assert st["world"] == 2
        with bdc.Engine(n, k, engine="count") as E:
            E.set_p(_start(n, spec))
            s1 = E.iterate(iters, a)
            p1 = E.get_p()
        assert st["iters"] == s1["iters"] and st["converged"] == bool(s1["converged"])
        np.testing.assert_allclose(p, p1, rtol=1e-12, atol=0)
        assert abs(st["upper_bound"] - s1["upper_bound"]) < 1e-12
        assert abs(st["rate"] - s1["rate"]) < 1e-12
        assert abs(st["mx"] - s1["mx"]) < 1e-11
    # the stopping case against the oracle's own loop (backend/main_BAA.cu:73)
    reps = O.canonicals(10)
    ref = O.run_ba(10, 5, np.full(len(reps), 1.0 / (1 << 10)), reps, 1e-3, 100000)
    assert res["stop"][0]["iters"] == ref["iters"]
