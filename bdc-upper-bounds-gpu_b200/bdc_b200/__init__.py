"""Host side of the B200 Blahut-Arimoto engine for the binary deletion channel.

Two layers, both over the C ABI of include/bdc_b200.h (libbdc_b200.so, built
in-tree by `make` in the package directory):

* ``Engine`` -- one handle per (n, k): device-resident iterate, ``iterate()``
  runs the BA loop on the device.
* module-level functions named and shaped like the reference host API
  (backend/BAA.cuh:21-29 and 295-362 of Pintz45/BDC-Upper-Bounds-GPU):
  ``load_cache``, ``baa_iteration``, ``compute_all_log_D``,
  ``compute_all_log_W``, ``compute_rate``, ``compute_max_deviation``, plus
  ``compute_C_n_k`` (backend/main_BAA.cu:39-131).  They take and return numpy
  vectors in the reference's layouts.

There is no CPU fallback: importing this module without the built library, or
using it on a machine without a CUDA device, raises.
"""
from __future__ import annotations

import ctypes
import os
import time

import numpy as np

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libbdc_b200.so")

BDC_OK = 0
STATUS_NAMES = {0: "OK", 1: "ERR_ARG", 2: "ERR_CUDA", 3: "ERR_IO", 4: "ERR_NOMEM",
                5: "ERR_STATE", 6: "ERR_UNSUPPORTED", 7: "ERR_NUMERIC"}
ENGINES = {"auto": 0, "count": 1, "factored": 2, "count-fp32c": 3}
ENGINE_NAMES = {v: k for k, v in ENGINES.items()}

# every symbol the C ABI exports (include/bdc_b200.h)
EXPORTED_SYMBOLS = [
    "bdc_default_options", "bdc_last_error", "bdc_version", "bdc_create", "bdc_destroy",
    "bdc_info", "bdc_get_reps", "bdc_set_p", "bdc_set_p_uniform", "bdc_get_p",
    "bdc_set_p_device", "bdc_get_p_device", "bdc_iterate", "bdc_baa_iteration", "bdc_log_q",
    "bdc_log_w", "bdc_divergence", "bdc_rate", "bdc_max_deviation", "bdc_counts",
    "bdc_generate_cache", "bdc_read_cache_file", "bdc_write_cache_file", "bdc_read_dist_file",
    "bdc_write_dist_file", "bdc_work", "bdc_profile", "bdc_set_stream", "bdc_peak_probe",
    "bdc_max_deviation_noalloc", "bdc_accelerate", "bdc_mi_forward", "bdc_mi_backward", "bdc_mi_backward_device",
    "bdc_batch_create", "bdc_batch_iterate", "bdc_batch_destroy", "bdc_batch_set_stream", "bdc_batch_accelerate",
    "bdc_create_sharded", "bdc_fshard_range", "bdc_fshard_q", "bdc_fshard_d", "bdc_fshard_finish", "bdc_fshard_get_p",
    "bdc_solve",
    "bdc_bound_error", "bdc_shard_q", "bdc_shard_set_q", "bdc_shard_update_begin", "bdc_shard_update_end",
]


class BDCError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {msg}")


class Options(ctypes.Structure):
    _fields_ = [("engine", ctypes.c_int), ("device", ctypes.c_int),
                ("cache_dir", ctypes.c_char_p), ("verbose", ctypes.c_int)]


class Profile(ctypes.Structure):
    _fields_ = [("ms_q", ctypes.c_double), ("ms_fold", ctypes.c_double), ("ms_d", ctypes.c_double),
                ("ms_update", ctypes.c_double), ("ms_iter", ctypes.c_double), ("ms_main", ctypes.c_double),
                ("work_main", ctypes.c_double), ("launches", ctypes.c_int), ("iters", ctypes.c_int),
                ("main_kind", ctypes.c_int), ("bytes_main", ctypes.c_double)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(ctypes.Structure):
    _fields_ = [("iters", ctypes.c_int64), ("total_iters", ctypes.c_int64), ("mx", ctypes.c_double),
                ("upper_bound", ctypes.c_double), ("rate", ctypes.c_double), ("lse", ctypes.c_double),
                ("best_upper_bound", ctypes.c_double), ("best_rate", ctypes.c_double),
                ("converged", ctypes.c_int)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_}


_u32p = ctypes.POINTER(ctypes.c_uint32)
_f64p = ctypes.POINTER(ctypes.c_double)
_lib = None


def library() -> ctypes.CDLL:
    """Load libbdc_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `make -C {PKG_DIR}` "
                          "(the engine has no CPU fallback)")
    L = ctypes.CDLL(LIB_PATH)
    st = ctypes.c_int
    h = ctypes.c_void_p
    L.bdc_default_options.argtypes = [ctypes.POINTER(Options)]
    L.bdc_default_options.restype = None
    L.bdc_last_error.restype = ctypes.c_char_p
    L.bdc_version.restype = ctypes.c_char_p
    L.bdc_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(Options), ctypes.POINTER(h)]
    L.bdc_destroy.argtypes = [h]
    L.bdc_info.argtypes = [h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                           ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
    L.bdc_get_reps.argtypes = [h, _u32p, ctypes.c_int64]
    L.bdc_set_p.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_set_p_uniform.argtypes = [h]
    L.bdc_get_p.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_set_p_device.argtypes = [h, ctypes.c_void_p, ctypes.c_int64]
    L.bdc_get_p_device.argtypes = [h, ctypes.c_void_p, ctypes.c_int64]
    L.bdc_iterate.argtypes = [h, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(Stats)]
    L.bdc_baa_iteration.argtypes = [h, _f64p, _f64p, ctypes.c_int64]
    L.bdc_accelerate.argtypes = [h, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(Stats)]
    L.bdc_solve.argtypes = [h, ctypes.c_double, ctypes.c_int64, ctypes.POINTER(Stats)]
    L.bdc_batch_create.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    L.bdc_batch_iterate.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(Stats)]
    L.bdc_batch_accelerate.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, ctypes.POINTER(Stats),
                                       _f64p]
    L.bdc_batch_destroy.argtypes = [ctypes.c_void_p]
    L.bdc_batch_set_stream.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
    L.bdc_mi_forward.argtypes = [h, _f64p, ctypes.c_int64, _f64p]
    L.bdc_mi_backward.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_mi_backward_device.argtypes = [h, ctypes.c_void_p, ctypes.c_int64]
    L.bdc_create_sharded.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(Options), ctypes.c_int, ctypes.c_int,
                                     ctypes.POINTER(h)]
    L.bdc_fshard_range.argtypes = [h, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                   ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]
    L.bdc_fshard_q.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_fshard_d.argtypes = [h, _f64p, ctypes.c_int64, _f64p]
    L.bdc_fshard_finish.argtypes = [h, _f64p, ctypes.c_double, ctypes.POINTER(Stats)]
    L.bdc_fshard_get_p.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_bound_error.argtypes = [h, _f64p, _f64p]
    L.bdc_shard_q.argtypes = [h, ctypes.c_int64, ctypes.c_int64, _f64p, ctypes.c_int64]
    L.bdc_shard_set_q.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_shard_update_begin.argtypes = [h, ctypes.c_int64, ctypes.c_int64, _f64p]
    L.bdc_shard_update_end.argtypes = [h, ctypes.c_int64, ctypes.c_int64, ctypes.c_double, _f64p]
    L.bdc_log_q.argtypes = [h, _f64p, ctypes.c_int64]
    L.bdc_log_w.argtypes = [h, _f64p, _f64p, ctypes.c_int64]
    L.bdc_divergence.argtypes = [h, _f64p, _f64p, ctypes.c_int64]
    L.bdc_rate.argtypes = [h, _f64p]
    L.bdc_max_deviation.argtypes = [h, _f64p, _f64p, ctypes.c_int64, _f64p]
    L.bdc_counts.argtypes = [h, _u32p, _u32p, ctypes.c_int64, _u32p]
    L.bdc_generate_cache.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _u32p]
    L.bdc_read_cache_file.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _u32p]
    L.bdc_write_cache_file.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, _u32p]
    L.bdc_read_dist_file.argtypes = [ctypes.c_char_p, _f64p, ctypes.c_int64,
                                     ctypes.POINTER(ctypes.c_int64)]
    L.bdc_write_dist_file.argtypes = [ctypes.c_char_p, _f64p, ctypes.c_int64]
    L.bdc_work.argtypes = [h, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int)]
    L.bdc_profile.argtypes = [h, ctypes.c_int, ctypes.POINTER(Profile)]
    L.bdc_set_stream.argtypes = [h, ctypes.c_void_p]
    L.bdc_max_deviation_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p,
                                            ctypes.c_void_p]
    L.bdc_peak_probe.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.POINTER(ctypes.c_double)]
    for name in EXPORTED_SYMBOLS:
        fn = getattr(L, name)
        if name not in ("bdc_default_options", "bdc_last_error", "bdc_version"):
            fn.restype = st
    _lib = L
    return L


def _check(rc: int, where: str) -> None:
    if rc != BDC_OK:
        msg = library().bdc_last_error()
        raise BDCError(rc, where, msg.decode() if msg else "")


def _f64(a, copy=False):
    a = np.array(a, dtype=np.float64, copy=copy, order="C") if copy else \
        np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_f64p)


def _u32(a):
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return a, a.ctypes.data_as(_u32p)


def nck(n: int, k: int) -> int:
    from math import comb
    return comb(n, k)


def num_q_slots(k: int) -> int:
    """Size of the ln q vector: 2^{k-1} rep-value slots (backend/BAA.cu:649-652)."""
    return (1 << (k - 1)) if k >= 1 else 1


class Engine:
    """One (n, k) BA problem resident on one GPU.

    engine: "auto" (fastest available), "count" (split-identity count path),
    "factored" (Kronecker-factored passes) or "count-fp32c" (the count path
    with its q and D sums in compensated FP32, n <= 26).  cache_dir:
    directory of cache_n_k files; None builds the half tables on the device.
    """

    def __init__(self, n: int, k: int, engine: str = "auto", device: int = 0,
                 cache_dir: str | None = None, verbose: bool = False, shard: tuple[int, int] | None = None):
        L = library()
        o = Options()
        L.bdc_default_options(ctypes.byref(o))
        o.engine = ENGINES[engine]
        o.device = device
        self._cache_dir = cache_dir.encode() if cache_dir else None
        o.cache_dir = self._cache_dir
        o.verbose = 1 if verbose else 0
        hdl = ctypes.c_void_p()
        if shard is None:
            _check(L.bdc_create(n, k, ctypes.byref(o), ctypes.byref(hdl)), "bdc_create")
        else:
            # the factored engine holding rank shard[0]'s window of the rows out of shard[1]
            _check(L.bdc_create_sharded(n, k, ctypes.byref(o), int(shard[0]), int(shard[1]), ctypes.byref(hdl)),
                   "bdc_create_sharded")
        self.shard = shard
        self._h = hdl
        self.n, self.k = n, k
        self.device = int(device)
        nn, kk, R, eng = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64(), ctypes.c_int()
        _check(L.bdc_info(self._h, ctypes.byref(nn), ctypes.byref(kk), ctypes.byref(R),
                          ctypes.byref(eng)), "bdc_info")
        self.R = int(R.value)
        self.engine = ENGINE_NAMES.get(eng.value, str(eng.value))
        self._reps = None

    # ----------------------------------------------------------- life cycle
    def close(self) -> None:
        if getattr(self, "_h", None):
            library().bdc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --------------------------------------------------------------- state
    @property
    def reps(self) -> np.ndarray:
        if self._reps is None:
            out = np.empty(self.R, dtype=np.uint32)
            _check(library().bdc_get_reps(self._h, out.ctypes.data_as(_u32p), self.R), "bdc_get_reps")
            self._reps = out
        return self._reps

    def set_p(self, p) -> None:
        p, pp = _f64(p)
        _check(library().bdc_set_p(self._h, pp, len(p)), "bdc_set_p")

    def set_uniform(self) -> None:
        _check(library().bdc_set_p_uniform(self._h), "bdc_set_p_uniform")

    def get_p(self) -> np.ndarray:
        out = np.empty(self.R, dtype=np.float64)
        _check(library().bdc_get_p(self._h, out.ctypes.data_as(_f64p), self.R), "bdc_get_p")
        return out

    def set_p_device(self, ptr: int) -> None:
        _check(library().bdc_set_p_device(self._h, ctypes.c_void_p(ptr), self.R), "bdc_set_p_device")

    def get_p_device(self, ptr: int) -> None:
        _check(library().bdc_get_p_device(self._h, ctypes.c_void_p(ptr), self.R), "bdc_get_p_device")

    # ----------------------------------------------------------- iteration
    def iterate(self, max_iters: int, a: float = float("-inf")) -> dict:
        """Run BA iterations on the device until mx < a or max_iters."""
        st = Stats()
        _check(library().bdc_iterate(self._h, int(max_iters), float(a), ctypes.byref(st)), "bdc_iterate")
        return st.as_dict()

    # ------------------------------------------------ one rank of sharded BA
    # ------------------------------------------- rows sharded (factored engine)
    def fshard_range(self) -> tuple[int, int, int, int]:
        """(first row, rows, first representative, end representative) held."""
        r0, rows, i0, i1 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int64(), ctypes.c_int64()
        _check(library().bdc_fshard_range(self._h, ctypes.byref(r0), ctypes.byref(rows), ctypes.byref(i0),
                                          ctypes.byref(i1)), "bdc_fshard_range")
        return r0.value, rows.value, int(i0.value), int(i1.value)

    def fshard_q(self) -> np.ndarray:
        out = np.empty(1 << self.k, dtype=np.float64)
        _check(library().bdc_fshard_q(self._h, out.ctypes.data_as(_f64p), len(out)), "bdc_fshard_q")
        return out

    def fshard_d(self, acc) -> np.ndarray:
        acc, pa = _f64(acc)
        out = np.empty(5, dtype=np.float64)
        _check(library().bdc_fshard_d(self._h, pa, len(acc), out.ctypes.data_as(_f64p)), "bdc_fshard_d")
        return out

    def fshard_finish(self, part5, a: float = float("-inf")) -> dict:
        part5, pp = _f64(part5)
        st = Stats()
        _check(library().bdc_fshard_finish(self._h, pp, float(a), ctypes.byref(st)), "bdc_fshard_finish")
        return st.as_dict()

    def fshard_get_p(self) -> np.ndarray:
        _, _, i0, i1 = self.fshard_range()
        out = np.empty(i1 - i0, dtype=np.float64)
        _check(library().bdc_fshard_get_p(self._h, out.ctypes.data_as(_f64p), len(out)), "bdc_fshard_get_p")
        return out

    def shard_q(self, r0: int, r1: int) -> np.ndarray:
        """Partial q sums of representatives [r0, r1): acc[y] over all 2^k y."""
        acc = np.empty(1 << self.k, dtype=np.float64)
        _check(library().bdc_shard_q(self._h, ctypes.c_int64(r0), ctypes.c_int64(r1), acc.ctypes.data_as(_f64p),
                                     ctypes.c_int64(len(acc))), "bdc_shard_q")
        return acc

    def shard_set_q(self, acc) -> None:
        acc = np.ascontiguousarray(acc, dtype=np.float64)
        _check(library().bdc_shard_set_q(self._h, acc.ctypes.data_as(_f64p), ctypes.c_int64(len(acc))),
               "bdc_shard_set_q")

    def shard_update_begin(self, r0: int, r1: int) -> np.ndarray:
        """[max logW, sum |O| exp(logW - max), max D, sum |O| p D, zero flag] on the shard."""
        st = np.empty(5, dtype=np.float64)
        _check(library().bdc_shard_update_begin(self._h, ctypes.c_int64(r0), ctypes.c_int64(r1),
                                                st.ctypes.data_as(_f64p)), "bdc_shard_update_begin")
        return st

    def shard_update_end(self, r0: int, r1: int, log_z: float) -> float:
        mx = ctypes.c_double()
        _check(library().bdc_shard_update_end(self._h, ctypes.c_int64(r0), ctypes.c_int64(r1),
                                              ctypes.c_double(log_z), ctypes.byref(mx)), "bdc_shard_update_end")
        return mx.value

    def bound_error(self) -> tuple[float, float]:
        """(|upper_bound - FP64|, |rate - FP64|) in bits for the last
        iteration: the compensated-FP32 engine's reported numbers against an
        FP64 re-evaluation at the same iterate; (0, 0) for the FP64 engines."""
        ub, rate = ctypes.c_double(), ctypes.c_double()
        _check(library().bdc_bound_error(self._h, ctypes.byref(ub), ctypes.byref(rate)), "bdc_bound_error")
        return ub.value, rate.value

    def accelerate(self, max_evals: int, gap_bits: float = 0.0) -> dict:
        """Nesterov-accelerated exponentiated gradient (adjoint-driven BA with
        momentum and adaptive restart) on the device (factored engine): runs
        until the bracket best_upper_bound - best_rate < gap_bits or
        max_evals evaluations."""
        st = Stats()
        _check(library().bdc_accelerate(self._h, int(max_evals), float(gap_bits), ctypes.byref(st)),
               "bdc_accelerate")
        return st.as_dict()

    def solve(self, gap_bits: float = 1e-9, max_evals: int = 100000) -> dict:
        """Certified bracket best_rate <= C <= best_upper_bound (bits) by
        accelerated BA, a restricted solve on the inputs that carry mass and a
        full-space check; the iterate becomes the final point."""
        st = Stats()
        _check(library().bdc_solve(self._h, float(gap_bits), int(max_evals), ctypes.byref(st)), "bdc_solve")
        return st.as_dict()

    def mi_forward(self, p=None) -> float:
        """I(p;W) in nats; p (per representative) becomes the current iterate."""
        r = ctypes.c_double()
        if p is None:
            _check(library().bdc_mi_forward(self._h, None, self.R, ctypes.byref(r)), "bdc_mi_forward")
        else:
            p, pp = _f64(p)
            _check(library().bdc_mi_forward(self._h, pp, len(p), ctypes.byref(r)), "bdc_mi_forward")
        return r.value

    def mi_backward(self) -> np.ndarray:
        """dI/dp per representative (nats) at the current iterate."""
        out = np.empty(self.R, dtype=np.float64)
        _check(library().bdc_mi_backward(self._h, out.ctypes.data_as(_f64p), self.R), "bdc_mi_backward")
        return out

    def mi_backward_device(self, ptr: int) -> None:
        """dI/dp per representative (nats) at the current iterate, written to
        the device buffer at `ptr` (R doubles on the handle's device)."""
        _check(library().bdc_mi_backward_device(self._h, ctypes.c_void_p(ptr), self.R), "bdc_mi_backward_device")

    def baa_iteration(self, p) -> np.ndarray:
        p, pp = _f64(p)
        out = np.empty(self.R, dtype=np.float64)
        _check(library().bdc_baa_iteration(self._h, pp, out.ctypes.data_as(_f64p), len(p)),
               "bdc_baa_iteration")
        return out

    # ------------------------------------------------------ single passes
    def log_q(self) -> np.ndarray:
        out = np.empty(num_q_slots(self.k), dtype=np.float64)
        _check(library().bdc_log_q(self._h, out.ctypes.data_as(_f64p), len(out)), "bdc_log_q")
        return out

    def log_w(self, lnq=None) -> np.ndarray:
        out = np.empty(self.R, dtype=np.float64)
        lp = None
        if lnq is not None:
            lnq, lp = _f64(lnq)
        _check(library().bdc_log_w(self._h, lp, out.ctypes.data_as(_f64p), self.R), "bdc_log_w")
        return out

    def divergence(self, lnq=None) -> np.ndarray:
        out = np.empty(self.R, dtype=np.float64)
        lp = None
        if lnq is not None:
            lnq, lp = _f64(lnq)
        _check(library().bdc_divergence(self._h, lp, out.ctypes.data_as(_f64p), self.R), "bdc_divergence")
        return out

    def rate(self) -> float:
        """I(p;W) in nats with a fresh q of the current p."""
        r = ctypes.c_double()
        _check(library().bdc_rate(self._h, ctypes.byref(r)), "bdc_rate")
        return r.value

    def max_deviation(self, p, p_before) -> float:
        p, pp = _f64(p)
        pb, pq = _f64(p_before)
        r = ctypes.c_double()
        _check(library().bdc_max_deviation(self._h, pp, pq, len(p), ctypes.byref(r)), "bdc_max_deviation")
        return r.value

    def work(self) -> tuple[int, int]:
        """(nonzero pairs per pass, split terms per pair)."""
        p, s = ctypes.c_int64(), ctypes.c_int()
        _check(library().bdc_work(self._h, ctypes.byref(p), ctypes.byref(s)), "bdc_work")
        return int(p.value), int(s.value)

    def set_stream(self, cuda_stream: int | None) -> None:
        """Queue work on a caller-owned cudaStream_t (an int handle); None
        returns to the handle's own stream."""
        _check(library().bdc_set_stream(self._h, ctypes.c_void_p(cuda_stream or 0)), "bdc_set_stream")

    def baa_iteration_ptr(self, p_in_ptr: int, p_out_ptr: int) -> None:
        """baa_iteration with host pointers (e.g. pinned buffers)."""
        _check(library().bdc_baa_iteration(self._h, ctypes.cast(p_in_ptr, _f64p),
                                           ctypes.cast(p_out_ptr, _f64p), self.R), "bdc_baa_iteration")

    def profile(self, iters: int) -> dict:
        """Per-pass CUDA-event times (ms) averaged over `iters` iterations."""
        pr = Profile()
        _check(library().bdc_profile(self._h, int(iters), ctypes.byref(pr)), "bdc_profile")
        return pr.as_dict()

    def counts(self, xs, ys) -> np.ndarray:
        xs, px = _u32(xs)
        ys, py = _u32(ys)
        if len(xs) != len(ys):
            raise ValueError("xs and ys differ in length")
        out = np.empty(len(xs), dtype=np.uint32)
        _check(library().bdc_counts(self._h, px, py, len(xs), out.ctypes.data_as(_u32p)), "bdc_counts")
        return out


class Batch:
    """Several engines (any mix of (n,k) and starting distributions) iterated
    together from one captured CUDA graph, one branch per engine."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (ctypes.c_void_p * len(self.engines))(*[E._h.value for E in self.engines])
        b = ctypes.c_void_p()
        _check(library().bdc_batch_create(arr, len(self.engines), ctypes.byref(b)), "bdc_batch_create")
        self._b = b

    def iterate(self, max_iters: int, a: float = float("-inf")) -> list:
        st = (Stats * len(self.engines))()
        _check(library().bdc_batch_iterate(self._b, int(max_iters), float(a), st), "bdc_batch_iterate")
        return [s.as_dict() for s in st]

    def accelerate(self, max_evals: int, gap_bits: float = 1e-9) -> tuple[list, list]:
        """The accelerated loop for every engine (factored), each stopping on
        its own bracket < gap_bits; returns (stats per engine, seconds per
        engine until its bracket fell below gap_bits, -1 if it did not)."""
        st = (Stats * len(self.engines))()
        sec = np.empty(len(self.engines), dtype=np.float64)
        _check(library().bdc_batch_accelerate(self._b, int(max_evals), float(gap_bits), st,
                                              sec.ctypes.data_as(_f64p)), "bdc_batch_accelerate")
        return [s.as_dict() for s in st], [float(v) for v in sec]

    def set_stream(self, stream: int | None) -> None:
        """Queue the batch's work on a cudaStream_t given as an integer handle."""
        _check(library().bdc_batch_set_stream(self._b, ctypes.c_void_p(stream or 0)), "bdc_batch_set_stream")

    def close(self) -> None:
        if getattr(self, "_b", None):
            library().bdc_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


# ------------------------------------------------------------ file formats
def generate_cache(n: int, k: int, device: int = 0) -> np.ndarray:
    """cache_{n,k} computed on the GPU (generate_bit_transition_cache.cpp:46-77)."""
    out = np.empty(1 << (n + k), dtype=np.uint32)
    _check(library().bdc_generate_cache(n, k, device, out.ctypes.data_as(_u32p)), "bdc_generate_cache")
    return out


def max_deviation_noalloc(p_ptr: int, p_before_ptr: int, num_reps: int, mx_ptr: int, stream: int = 0) -> None:
    """Allocation-free max_i log2 p - log2 p_before over caller-owned device
    arrays (raw device pointers), result written to the device double at
    mx_ptr.  For callers whose device memory all comes from their own pool:
    the library allocates nothing here and uses one fixed scratch array per
    device instead (num_reps <= 2^27; overlapping calls on the GPU race)."""
    _check(library().bdc_max_deviation_noalloc(ctypes.c_void_p(p_ptr), ctypes.c_void_p(p_before_ptr),
                                               int(num_reps), ctypes.c_void_p(mx_ptr), ctypes.c_void_p(stream)),
           "bdc_max_deviation_noalloc")


def peak_probe(kind: str, device: int = 0, ms: float = 50.0) -> float:
    """Measured multiply-adds/s of one arithmetic path: "imad", "dfma",
    "ffma" or "dmma" (FP64 mma.sync)."""
    r = ctypes.c_double()
    _check(library().bdc_peak_probe(device, {"imad": 0, "dfma": 1, "ffma": 2, "dmma": 3}[kind], ms, ctypes.byref(r)),
           "bdc_peak_probe")
    return r.value


def read_cache_file(path: str, n: int, k: int) -> np.ndarray:
    out = np.empty(1 << (n + k), dtype=np.uint32)
    _check(library().bdc_read_cache_file(path.encode(), n, k, out.ctypes.data_as(_u32p)),
           "bdc_read_cache_file")
    return out


def write_cache_file(path: str, n: int, k: int, data) -> None:
    data, pd = _u32(data)
    if len(data) != 1 << (n + k):
        raise ValueError("cache size is not 2^(n+k)")
    _check(library().bdc_write_cache_file(path.encode(), n, k, pd), "bdc_write_cache_file")


def read_dist_file(path: str) -> np.ndarray:
    L = library()
    cnt = ctypes.c_int64()
    _check(L.bdc_read_dist_file(path.encode(), None, 0, ctypes.byref(cnt)), "bdc_read_dist_file")
    out = np.empty(cnt.value, dtype=np.float64)
    _check(L.bdc_read_dist_file(path.encode(), out.ctypes.data_as(_f64p), cnt.value, ctypes.byref(cnt)),
           "bdc_read_dist_file")
    return out


def write_dist_file(path: str, p) -> None:
    p, pp = _f64(p)
    _check(library().bdc_write_dist_file(path.encode(), pp, len(p)), "bdc_write_dist_file")


def cache_filename(n: int, k: int, base: str = ".") -> str:
    """./transition_counts/cache_n_k (backend/cache_io.h:7-14)."""
    return os.path.join(base, "transition_counts", f"cache_{n}_{k}")


def dist_filename(n: int, k: int, base: str = ".") -> str:
    """distributions/dist_n_k.txt (backend/main_BAA.cu:55-57)."""
    return os.path.join(base, "distributions", f"dist_{n}_{k}.txt")


# ------------------------------------------- reference-shaped host API
_default: Engine | None = None


def load_cache(n: int, k: int, cache_dir: str | None = "transition_counts",
               engine: str = "auto", device: int = 0) -> Engine:
    """load_cache (backend/BAA.cu:183-188): one (n, k) per process.  Reads
    cache_dir/cache_{h}_{m} like the reference; cache_dir=None builds the
    tables on the device instead."""
    global _default
    if _default is not None:
        _default.close()
    _default = Engine(n, k, engine=engine, device=device, cache_dir=cache_dir)
    return _default


def _engine_for(n: int, k: int, trans_canonicals) -> Engine:
    if _default is None or _default.n != n or _default.k != k:
        raise BDCError(5, "reference API", f"load_cache({n}, {k}) has not been called")
    if trans_canonicals is not None and len(trans_canonicals) != _default.R:
        raise BDCError(1, "reference API", "trans_canonicals is not the canonical list")
    return _default


def baa_iteration(Q_i, trans_canonicals, n: int, k: int) -> np.ndarray:
    """backend/BAA.cu:590-639: one BA step, returns the new distribution."""
    return _engine_for(n, k, trans_canonicals).baa_iteration(Q_i)


def compute_all_log_D(Q_i, trans_canonicals, n: int, k: int) -> np.ndarray:
    """backend/BAA.cu:642-724: ln q over the 2^{k-1} rep-value slots."""
    E = _engine_for(n, k, trans_canonicals)
    E.set_p(Q_i)
    return E.log_q()


def compute_all_log_W(Q_i, log_den, trans_canonicals, n: int, k: int) -> np.ndarray:
    """backend/BAA.cu:727-814: ln p + D per representative."""
    E = _engine_for(n, k, trans_canonicals)
    E.set_p(Q_i)
    return E.log_w(log_den)


def compute_rate(log_den, Q_i, trans_canonicals, n: int, k: int) -> float:
    """backend/BAA.cu:836-913: sum |O| p KL in nats, KL from the given ln q."""
    E = _engine_for(n, k, trans_canonicals)
    E.set_p(Q_i)
    kl = E.divergence(log_den)
    orb = orbit_sizes(E.reps, n)
    return float(np.sum(orb * np.asarray(Q_i, dtype=np.float64) * kl))


def compute_max_deviation(Q, Q_before) -> float:
    """backend/BAA.cu:916-946: max log2 Q - log2 Q_before (on the device)."""
    if _default is None:
        raise BDCError(5, "compute_max_deviation", "load_cache has not been called")
    return _default.max_deviation(Q, Q_before)


def orbit_sizes(xs, n: int) -> np.ndarray:
    """|orbit| (2 or 4) of each n-bit string (backend/BAA.cu:230-241)."""
    xs = np.asarray(xs, dtype=np.uint64)
    r = reverse_bits(xs, n)
    rc = reverse_bits(xs ^ np.uint64((1 << n) - 1), n)
    return np.where((xs == r) | (xs == rc), 2.0, 4.0)


_REV8 = np.array([int(f"{i:08b}"[::-1], 2) for i in range(256)], dtype=np.uint64)


def reverse_bits(xs, n: int) -> np.ndarray:
    """Bit reversal of n-bit strings (n <= 32), a byte at a time."""
    xs = np.asarray(xs, dtype=np.uint64)
    b = np.uint64(0xFF)
    r = ((_REV8[xs & b] << np.uint64(24)) | (_REV8[(xs >> np.uint64(8)) & b] << np.uint64(16))
         | (_REV8[(xs >> np.uint64(16)) & b] << np.uint64(8)) | _REV8[(xs >> np.uint64(24)) & b])
    return r >> np.uint64(32 - n) if n > 0 else np.zeros_like(xs)


def canonical_reps(n: int) -> np.ndarray:
    """Ascending canonical representatives (backend/main_BAA.cu:46-50), host."""
    x = np.arange(1 << n, dtype=np.uint64)
    m = np.uint64((1 << n) - 1)
    r = reverse_bits(x, n)
    c = x ^ m
    rc = reverse_bits(c, n)
    rep = np.minimum(np.minimum(x, r), np.minimum(c, rc))
    return x[rep == x].astype(np.uint32)


def compute_C_n_k(in_len: int, out_len: int, a: float = 0.005, read_from_file: bool = False,
                  save_iterations: int = 100, base: str = ".", engine: str = "auto",
                  cache_dir: str | None = "transition_counts", verbose: bool = True,
                  max_iters: int | None = None, certified_gap: float | None = None) -> dict:
    """backend/main_BAA.cu:39-131: BA until mx < a, saving the distribution
    every save_iterations and at the end; returns rate (bits) and mx.  With
    certified_gap (bits) the certified solver replaces the loop and the result
    also holds the bracket lower_bits <= C <= upper_bits."""
    E = load_cache(in_len, out_len, cache_dir=os.path.join(base, cache_dir) if cache_dir else None,
                   engine=engine)
    path = dist_filename(in_len, out_len, base)
    if read_from_file:
        if verbose:
            print(f"Loading distribution from file: {os.path.relpath(path, base)}")
        E.set_p(read_dist_file(path))
    else:
        if verbose:
            print("Initializing uniform distribution")
        E.set_uniform()
    if certified_gap is not None:
        t0 = time.perf_counter()
        st = E.solve(certified_gap, 1000000)
        p = E.get_p()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        write_dist_file(path, p)
        if verbose:
            print(f"Certified C_{{{in_len},{out_len}}} in [{st['best_rate']:.15f}, {st['best_upper_bound']:.15f}] bits")
        return {"rate_bits": st["best_rate"], "lower_bits": st["best_rate"], "upper_bits": st["best_upper_bound"],
                "converged": bool(st["converged"]), "iters": st["iters"], "p": p,
                "loop_s": time.perf_counter() - t0}
    if verbose:
        print("Starting BAA iterations...")
    i = 0
    mx = a
    t_loop = time.perf_counter()
    while mx >= a and (max_iters is None or i < max_iters):
        chunk = save_iterations - (i % save_iterations)
        if max_iters is not None:
            chunk = min(chunk, max_iters - i)
        t0 = time.perf_counter()
        st = E.iterate(chunk, a)
        dt = time.perf_counter() - t0
        i += st["iters"]
        mx = st["mx"]
        if verbose:
            print(f"Iteration {i}: mx = {mx:.6f}, time = {dt / max(st['iters'], 1):.3f} s")
        if i % save_iterations == 0 and st["iters"] > 0:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            write_dist_file(path, E.get_p())
    os.makedirs(os.path.dirname(path), exist_ok=True)
    p = E.get_p()
    write_dist_file(path, p)
    if verbose:
        print(f"Final distribution saved to {os.path.relpath(path, base)}")
    rate_bits = E.rate() / np.log(2.0)
    if verbose:
        print(f"Computed C_{{{in_len},{out_len}}} = {rate_bits:.6f} bits (max deviation {mx:.6f})")
    return {"rate_bits": rate_bits, "mx": mx, "iters": i, "p": p,
            "loop_s": time.perf_counter() - t_loop}
