"""ctypes wrapper of the CPU oracle (liboracle.so, built from bdc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference legs of bench.py as the checker.  The product never
imports this module.

Each function mirrors one reference function; see the citations in
bdc_oracle.c (backend/BAA.cu, backend/main_BAA.cu,
backend/generate_bit_transition_cache.cpp of Pintz45/BDC-Upper-Bounds-GPU).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None


def build() -> None:
    """Compile liboracle.so (and, when the reference sources exist, _ref/)."""
    subprocess.run(["make", "-s", "liboracle.so"], cwd=HERE, check=True)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_nck.restype = ctypes.c_uint32
        L.oracle_nck.argtypes = [ctypes.c_uint32, ctypes.c_uint32]
        L.oracle_rep.restype = ctypes.c_uint32
        L.oracle_rep.argtypes = [ctypes.c_uint32, ctypes.c_int]
        L.oracle_orbit.restype = ctypes.c_int
        L.oracle_orbit.argtypes = [ctypes.c_uint32, ctypes.c_int]
        L.oracle_canonicals.restype = ctypes.c_int64
        L.oracle_canonicals.argtypes = [ctypes.c_int, _u32p, ctypes.c_int64]
        L.oracle_count_dp.restype = ctypes.c_uint32
        L.oracle_count_dp.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_uint32, ctypes.c_int]
        L.oracle_gen_cache.restype = None
        L.oracle_gen_cache.argtypes = [ctypes.c_int, ctypes.c_int, _u32p]
        L.oracle_num_distinct.restype = ctypes.c_uint32
        L.oracle_num_distinct.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
        L.oracle_distinct_subsequences.restype = ctypes.c_uint32
        L.oracle_distinct_subsequences.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_int, _u32p]
        L.oracle_total_transitions.restype = ctypes.c_uint32
        L.oracle_total_transitions.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.c_int]
        L.oracle_counts_pairs.restype = None
        L.oracle_counts_pairs.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, _u32p, ctypes.c_int64, _u32p]
        L.oracle_count_rows.restype = None
        L.oracle_count_rows.argtypes = [ctypes.c_int, ctypes.c_int, _u32p, ctypes.c_int64, _u32p]
        L.oracle_log_q.restype = None
        L.oracle_log_q.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _u32p, ctypes.c_int64, _f64p]
        L.oracle_log_w.restype = None
        L.oracle_log_w.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _f64p, _u32p, ctypes.c_int64, _f64p]
        L.oracle_kl.restype = None
        L.oracle_kl.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _u32p, ctypes.c_int64, _f64p]
        L.oracle_normalise.restype = None
        L.oracle_normalise.argtypes = [ctypes.c_int, _f64p, _u32p, ctypes.c_int64, _f64p]
        L.oracle_ba_iteration.restype = None
        L.oracle_ba_iteration.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _u32p, ctypes.c_int64,
                                          _f64p, _f64p, _f64p]
        L.oracle_max_deviation.restype = ctypes.c_double
        L.oracle_max_deviation.argtypes = [_f64p, _f64p, ctypes.c_int64]
        L.oracle_rate.restype = ctypes.c_double
        L.oracle_rate.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _f64p, _u32p, ctypes.c_int64]
        L.oracle_run_ba.restype = ctypes.c_int64
        L.oracle_run_ba.argtypes = [ctypes.c_int, ctypes.c_int, _f64p, _u32p, ctypes.c_int64,
                                    ctypes.c_double, ctypes.c_int64, _f64p, _f64p, _f64p, _f64p]
        L.oracle_set_threads.restype = None
        L.oracle_set_threads.argtypes = [ctypes.c_int]
        L.oracle_get_threads.restype = ctypes.c_int
        L.oracle_get_threads.argtypes = []
        _lib = L
    return _lib


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(_u32p)


def _f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_f64p)


def set_threads(t: int) -> None:
    lib().oracle_set_threads(int(t))


def threads() -> int:
    return int(lib().oracle_get_threads())


def nck(n: int, k: int) -> int:
    return int(lib().oracle_nck(n, k))


def rep(x: int, length: int) -> int:
    return int(lib().oracle_rep(x, length))


def orbit(x: int, length: int) -> int:
    return int(lib().oracle_orbit(x, length))


def canonicals(n: int) -> np.ndarray:
    L = lib()
    cnt = L.oracle_canonicals(n, None, 0)
    out = np.empty(cnt, dtype=np.uint32)
    L.oracle_canonicals(n, out.ctypes.data_as(_u32p), cnt)
    return out


def orbits_of(xs: np.ndarray, length: int) -> np.ndarray:
    L = lib()
    return np.array([L.oracle_orbit(int(x), length) for x in xs], dtype=np.float64)


def count_dp(x: int, n: int, y: int, k: int) -> int:
    return int(lib().oracle_count_dp(x, n, y, k))


def gen_cache(n: int, k: int) -> np.ndarray:
    out = np.empty(1 << (n + k), dtype=np.uint32)
    lib().oracle_gen_cache(n, k, out.ctypes.data_as(_u32p))
    return out


def distinct_subsequences(x: int, n: int, k: int) -> np.ndarray:
    L = lib()
    c = L.oracle_num_distinct(x, n, k)
    out = np.empty(max(c, 1), dtype=np.uint32)
    L.oracle_distinct_subsequences(x, n, k, out.ctypes.data_as(_u32p))
    return out[:c]


def total_transitions(x: int, y: int, n: int, k: int) -> int:
    return int(lib().oracle_total_transitions(x, y, n, k))


def counts_pairs(n: int, k: int, xs, ys) -> np.ndarray:
    xs, px = _u32(xs)
    ys, py = _u32(ys)
    out = np.empty(len(xs), dtype=np.uint32)
    lib().oracle_counts_pairs(n, k, px, py, len(xs), out.ctypes.data_as(_u32p))
    return out


def count_rows(n: int, k: int, xs) -> np.ndarray:
    xs, px = _u32(xs)
    out = np.empty((len(xs), 1 << k), dtype=np.uint32)
    lib().oracle_count_rows(n, k, px, len(xs), out.ctypes.data_as(_u32p))
    return out


def nq(k: int) -> int:
    return (1 << (k - 1)) if k >= 1 else 1


def log_q(n: int, k: int, p, reps) -> np.ndarray:
    p, pp = _f64(p)
    reps, pr = _u32(reps)
    out = np.empty(nq(k), dtype=np.float64)
    lib().oracle_log_q(n, k, pp, pr, len(reps), out.ctypes.data_as(_f64p))
    return out


def log_w(n: int, k: int, p, lnq, reps) -> np.ndarray:
    p, pp = _f64(p)
    lnq, pq = _f64(lnq)
    reps, pr = _u32(reps)
    out = np.empty(len(reps), dtype=np.float64)
    lib().oracle_log_w(n, k, pp, pq, pr, len(reps), out.ctypes.data_as(_f64p))
    return out


def kl(n: int, k: int, lnq, reps) -> np.ndarray:
    lnq, pq = _f64(lnq)
    reps, pr = _u32(reps)
    out = np.empty(len(reps), dtype=np.float64)
    lib().oracle_kl(n, k, pq, pr, len(reps), out.ctypes.data_as(_f64p))
    return out


def normalise(n: int, logw, reps) -> np.ndarray:
    logw, pl = _f64(logw)
    reps, pr = _u32(reps)
    out = np.empty(len(reps), dtype=np.float64)
    lib().oracle_normalise(n, pl, pr, len(reps), out.ctypes.data_as(_f64p))
    return out


def ba_iteration(n: int, k: int, p, reps):
    """Returns (p_next, lnq, logw) of one reference BA iteration."""
    p, pp = _f64(p)
    reps, pr = _u32(reps)
    pn = np.empty(len(reps), dtype=np.float64)
    lnq = np.empty(nq(k), dtype=np.float64)
    lw = np.empty(len(reps), dtype=np.float64)
    lib().oracle_ba_iteration(n, k, pp, pr, len(reps), pn.ctypes.data_as(_f64p),
                              lnq.ctypes.data_as(_f64p), lw.ctypes.data_as(_f64p))
    return pn, lnq, lw


def max_deviation(p, pb) -> float:
    p, pp = _f64(p)
    pb, pq = _f64(pb)
    return float(lib().oracle_max_deviation(pp, pq, len(p)))


def rate(n: int, k: int, lnq, p, reps) -> float:
    """I(p;W) in nats."""
    lnq, pq = _f64(lnq)
    p, pp = _f64(p)
    reps, pr = _u32(reps)
    return float(lib().oracle_rate(n, k, pq, pp, pr, len(reps)))


def run_ba(n: int, k: int, p0, reps, a: float, max_iters: int):
    """The reference outer loop (main_BAA.cu:39-131).  Returns a dict with the
    final p, iterations, per-iteration mx and upper bound (bits), final rate
    (bits) and final mx."""
    p, pp = _f64(np.array(p0, dtype=np.float64, copy=True))
    reps, pr = _u32(reps)
    mxl = np.full(max_iters, np.nan)
    ubl = np.full(max_iters, np.nan)
    rb = ctypes.c_double(0.0)
    mf = ctypes.c_double(0.0)
    it = lib().oracle_run_ba(n, k, pp, pr, len(reps), a, max_iters,
                             mxl.ctypes.data_as(_f64p), ubl.ctypes.data_as(_f64p),
                             ctypes.byref(rb), ctypes.byref(mf))
    return {"p": p, "iters": int(it), "mx": mxl[:it], "ub_bits": ubl[:it],
            "rate_bits": rb.value, "mx_final": mf.value}
