"""BA sharded by input strings over several GPUs (no counterpart in the
reference, which runs one (n,k) on one GPU: backend/main_BAA.cu:39-131).

One process per GPU.  Rank r holds a count-engine handle for the whole (n,k),
sets the same starting distribution as every other rank, and owns the
contiguous range shard_range(R, r, world) of the representatives: the q pass,
the D pass and the update touch p only there.  Per iteration the ranks
exchange
  * the 2^k partial q sums (one all-reduce of 2^k doubles),
  * the update's shift and the bound (one max all-reduce of two values), then
    the normaliser and the rate (one sum all-reduce of two values),
  * the stopping statistic mx (one max all-reduce),
over torch.distributed: NCCL with tensors on the handle's own GPU, gloo with
CPU tensors.  The combination of the per-rank update statistics is in
combine_update, a pure function.

The handle's own single-GPU statistics (bdc_iterate's bound, rate and mx) are
not the sharded problem's after a sharded iteration: use what iterate()
returns."""
from __future__ import annotations

import math

import numpy as np

LN2 = math.log(2.0)


def shard_range(R: int, rank: int, world: int) -> tuple[int, int]:
    """Representatives [r0, r1) of rank `rank` out of `world` (contiguous,
    sizes differing by at most one)."""
    if world < 1 or not 0 <= rank < world or R < world:
        raise ValueError(f"cannot shard {R} representatives over {world} ranks (rank {rank})")
    return R * rank // world, R * (rank + 1) // world


def z_share(z_r: float, shift_r: float, S: float) -> float:
    """Rank r's term of the global normaliser, Z_r exp(s_r - S)."""
    return z_r * math.exp(shift_r - S) if z_r > 0 else 0.0


def combine_update(shift, z) -> tuple[float, float]:
    """Global (S, ln Z) from per-rank shifts s_r = max logW on the shard and
    normalisers Z_r = sum |O| exp(logW - s_r): S = max s_r and
    Z = sum_r Z_r exp(s_r - S), so that p' = exp(logW - s_r) / exp(ln Z + S - s_r)
    on every shard (what iterate computes with two all-reduces)."""
    S = float(max(shift))
    return S, math.log(sum(z_share(float(zr), float(sr), S) for zr, sr in zip(z, shift)))


def shard_log_z(S: float, log_z: float, shift_r: float) -> float:
    """The normaliser that rank r passes to bdc_shard_update_end."""
    return log_z + S - shift_r


def comm_device(backend: str, device: int) -> str:
    """Where a rank's exchange tensors live: NCCL needs them on the rank's
    own GPU (the handle's device, which need not be torch's current device),
    gloo on the host."""
    return f"cuda:{int(device)}" if backend == "nccl" else "cpu"


class _Comm:
    def __init__(self, group=None, device: int = 0):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = comm_device(dist.get_backend(group), device)

    def reduce(self, vals, op: str) -> np.ndarray:
        t = self.torch.tensor(np.asarray(vals, dtype=np.float64), device=self.device)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM,
                             group=self.group)
        return t.cpu().numpy()


def iterate(E, max_iters: int, a: float = float("-inf"), group=None) -> dict:
    """BA iterations of a count-engine handle sharded over the ranks of
    `group` (torch.distributed, initialised by the caller), until the global
    mx < a or max_iters; every rank returns the same statistics (bits)."""
    comm = _Comm(group, E.device)
    r0, r1 = shard_range(E.R, comm.rank, comm.world)
    out = {"iters": 0, "mx": float("nan"), "upper_bound": float("nan"), "rate": float("nan"),
           "best_upper_bound": float("inf"), "best_rate": float("-inf"), "converged": False,
           "shard": (r0, r1), "world": comm.world}
    for _ in range(int(max_iters)):
        acc = comm.reduce(E.shard_q(r0, r1), "sum")
        E.shard_set_q(acc)
        st = E.shard_update_begin(r0, r1)
        S, max_d = (float(v) for v in comm.reduce([st[0], st[2]], "max"))
        z_rate = comm.reduce([z_share(st[1], st[0], S), st[3]], "sum")
        mx = E.shard_update_end(r0, r1, shard_log_z(S, math.log(z_rate[0]), st[0]))
        mx = float(comm.reduce([mx], "max")[0])
        out["iters"] += 1
        out["mx"] = mx
        out["upper_bound"] = max_d / LN2
        out["rate"] = float(z_rate[1]) / LN2
        out["best_upper_bound"] = min(out["best_upper_bound"], out["upper_bound"])
        out["best_rate"] = max(out["best_rate"], out["rate"])
        if not mx >= a:  # the reference's loop condition, main_BAA.cu:73
            out["converged"] = True
            break
    return out


def combine_part5(parts) -> np.ndarray:
    """The update statistics of row shards combined: [max D, sum |O| e,
    max logW, sum |O| p D, input-zero flag] -> max, sum, max, sum, max."""
    P = np.asarray(parts, dtype=np.float64).reshape(-1, 5)
    return np.array([P[:, 0].max(), P[:, 1].sum(), P[:, 2].max(), P[:, 3].sum(), P[:, 4].max()])


def iterate_rows(E, max_iters: int, a: float = float("-inf"), group=None) -> dict:
    """BA iterations of a factored-engine handle created with shard=(rank,
    world) (each rank holds a window of whole rows of the dense iterate),
    until mx < a or max_iters.  Per iteration: one sum all-reduce of the 2^k
    partial q sums, then one max all-reduce of [max D, max logW, zero flag]
    and one sum all-reduce of [sum |O| e, sum |O| p D] (the shift that scales
    e is the same on every rank).  Every rank returns the same statistics
    (bits)."""
    comm = _Comm(group, E.device)
    out = {"iters": 0, "world": comm.world, "rows": E.fshard_range()}
    for _ in range(int(max_iters)):
        acc = comm.reduce(E.fshard_q(), "sum")
        part = E.fshard_d(acc)
        mx3 = comm.reduce([part[0], part[2], part[4]], "max")
        sm2 = comm.reduce([part[1], part[3]], "sum")
        st = E.fshard_finish([mx3[0], sm2[0], mx3[1], sm2[1], mx3[2]], a)
        out["iters"] += 1
        out.update({key: st[key] for key in ("mx", "upper_bound", "rate", "best_upper_bound", "best_rate")})
        out["converged"] = bool(st["converged"])
        if out["converged"]:
            break
    return out


def gather_p_rows(E, group=None) -> np.ndarray | None:
    """The iterate of a row-sharded handle assembled on rank 0 (None elsewhere)."""
    comm = _Comm(group, E.device)
    _, _, i0, i1 = E.fshard_range()
    parts = [None] * comm.world
    comm.dist.all_gather_object(parts, (i0, E.fshard_get_p()), group=group)
    if comm.rank != 0:
        return None
    p = np.empty(E.R, dtype=np.float64)
    for lo, v in parts:
        p[lo:lo + len(v)] = v
    return p


def gather_p(E, group=None) -> np.ndarray | None:
    """The sharded iterate, assembled on rank 0 (None elsewhere)."""
    comm = _Comm(group, E.device)
    r0, r1 = shard_range(E.R, comm.rank, comm.world)
    mine = (r0, E.get_p()[r0:r1])
    parts = [None] * comm.world
    comm.dist.all_gather_object(parts, mine, group=group)
    if comm.rank != 0:
        return None
    p = np.empty(E.R, dtype=np.float64)
    for lo, v in parts:
        p[lo:lo + len(v)] = v
    return p
