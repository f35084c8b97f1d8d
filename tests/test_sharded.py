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


# ------------------------------------- the factored engine, rows sharded
def test_combine_part5_is_max_sum_max_sum_max():
    from bdc_b200 import sharded
    parts = [[1.0, 2.0, -3.0, 0.5, 0.0], [4.0, 1.0, -5.0, 0.25, 1.0], [2.0, 0.5, -1.0, 0.0, 0.0]]
    np.testing.assert_array_equal(sharded.combine_part5(parts), [4.0, 3.5, -1.0, 0.75, 1.0])


class _RowShardStandIn:
    """The three calls of a row-sharded factored handle restated in numpy on
    the full input space (every orbit of size one), for testing the exchange
    logic of sharded.iterate_rows without a GPU: fshard_q returns the held
    rows' partial sums acc[y] = sum_x e(x) N(x, y), fshard_d the update
    statistics of the held rows with the shift every rank shares, and
    fshard_finish the normaliser, the stopping statistic and the next shift
    from the combined statistics (the device finalize's arithmetic)."""

    def __init__(self, n, k, rank, world, p0, O):
        xs = np.arange(1 << n, dtype=np.uint32)
        self.N = O.count_rows(n, k, xs).reshape(1 << n, 1 << k).astype(np.float64)
        self.C = float(O.nck(n, k))
        W = self.N / self.C
        self.h = np.where(W > 0, W * np.log(np.where(W > 0, W, 1.0)), 0.0).sum(1)
        self.k, self.R, self.device = k, 1 << n, 0
        self.i0, self.i1 = (1 << n) * rank // world, (1 << n) * (rank + 1) // world
        self.lt = np.log(p0)                 # ln e (unnormalised), all rows (only held ones are used)
        self.log_z, self.shift = 0.0, float(np.log(p0).max()) + k * np.log(2.0)

    def fshard_range(self):
        return (self.i0, self.i1 - self.i0, self.i0, self.i1)

    def fshard_q(self):
        sl = slice(self.i0, self.i1)
        return np.exp(self.lt[sl] - self.log_z) @ self.N[sl]

    def fshard_d(self, acc):
        sl = slice(self.i0, self.i1)
        q = acc / self.C
        lnq = np.log(np.where(q > 0, q, 1.0))
        D = self.h[sl] - (self.N[sl] @ lnq) / self.C
        p = np.exp(self.lt[sl] - self.log_z)
        lw = (self.lt[sl] - self.log_z) + D - self.shift
        self.lt[sl] = lw
        return np.array([D.max(), np.exp(lw).sum(), lw.max(), (p * D).sum(), 0.0])

    def fshard_finish(self, part5, a):
        mD, sE, mL, sR, _ = part5
        lnz = np.log(sE)
        mx = (mD - self.shift - lnz) / np.log(2.0)
        # ln e carries the shift: ln p = lt - ln Z from here on
        self.shift, self.log_z = (mL - lnz) + mD, lnz
        return {"mx": mx, "upper_bound": mD / np.log(2.0), "rate": sR / np.log(2.0),
                "best_upper_bound": mD / np.log(2.0), "best_rate": sR / np.log(2.0), "converged": not mx >= a}

    def p(self):
        return np.exp(self.lt - self.log_z)


def _rows_rank(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(PKG), "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle as O
        from bdc_b200 import sharded
        n, k = 8, 4
        p0 = np.random.default_rng(3).dirichlet(np.ones(1 << n))
        E = _RowShardStandIn(n, k, rank, world, p0, O)
        st = sharded.iterate_rows(E, 25, float("-inf"))
        parts = [None] * world
        dist.all_gather_object(parts, (E.i0, E.p()[E.i0:E.i1]))
        if rank == 0:
            p = np.concatenate([v for _, v in sorted(parts, key=lambda t: t[0])])
            q.put((st, p))
    finally:
        dist.destroy_process_group()


def test_row_shards_over_gloo_world_2_match_one_process(O):
    # the same 25 BA iterations on the full space of n = 8 in one process
    n, k = 8, 4
    p = np.random.default_rng(3).dirichlet(np.ones(1 << n))
    N = O.count_rows(n, k, np.arange(1 << n, dtype=np.uint32)).reshape(1 << n, 1 << k).astype(np.float64)
    W = N / O.nck(n, k)
    for _ in range(25):
        qv = p @ W
        D = (W * np.log(np.where(W > 0, W / qv, 1.0))).sum(1)
        bound, rate = D.max() / np.log(2.0), (p * D).sum() / np.log(2.0)
        pn = p * np.exp(D)
        pn /= pn.sum()
        mx = np.max(np.log2(pn) - np.log2(p))
        p = pn
    ctx = mp.get_context("spawn")
    qq = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rows_rank, args=(r, 2, port, qq)) for r in range(2)]
    for pr in procs:
        pr.start()
    st, got = qq.get(timeout=120)
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    assert st["iters"] == 25 and st["world"] == 2
    np.testing.assert_allclose(got, p, rtol=1e-12, atol=0)
    assert abs(st["upper_bound"] - bound) < 1e-12 and abs(st["rate"] - rate) < 1e-12
    assert abs(st["mx"] - mx) < 1e-10


ROW_CASES = [(20, 10, ("dirichlet", 1.0, 0), 12), (24, 12, ("uniform",), 6)]


def _gpu_rows_rank(rank, world, port, q):
    import sys
    sys.path.insert(0, PKG)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=300))
    try:
        import bdc_b200
        from bdc_b200 import sharded
        res = {}
        for n, k, spec, iters in ROW_CASES:
            with bdc_b200.Engine(n, k, engine="factored", device=0, shard=(rank, world)) as E:
                E.set_p(_start(n, spec))
                st = sharded.iterate_rows(E, iters)
                p = sharded.gather_p_rows(E)
            res[(n, k)] = (st, p)
        if rank == 0:
            q.put(res)
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_row_sharded_factored_engine_two_ranks_match_one_engine(bdc):
    # two ranks, each holding half of the representatives' rows, as two
    # processes on one device exchanging over gloo (no kernel waits on another)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_rows_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=600)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    for n, k, spec, iters in ROW_CASES:
        st, p = res[(n, k)]
        assert st["world"] == 2 and st["iters"] == iters
        with bdc.Engine(n, k, engine="factored") as E:
            E.set_p(_start(n, spec))
            s1 = E.iterate(iters, float("-inf"))
            p1 = E.get_p()
        np.testing.assert_allclose(p, p1, rtol=1e-11, atol=0)
        assert abs(st["upper_bound"] - s1["upper_bound"]) < 1e-11
        assert abs(st["rate"] - s1["rate"]) < 1e-11
        assert abs(st["mx"] - s1["mx"]) < 1e-10
