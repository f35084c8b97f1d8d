"""Distribution tooling: seeded starting distributions and orbit bookkeeping.

A distribution over {0,1}^n is stored like the reference stores it
(backend/main_BAA.cu:46-64, README "Structure of Distribution Files"): one
value per canonical representative in ascending order, each value being the
probability of every string of that orbit, so that sum |O(rep)| p(rep) = 1.

Pure numpy; does not load the CUDA library.
"""
from __future__ import annotations

import numpy as np

from . import canonical_reps, orbit_sizes, reverse_bits


def rep_of(xs, n: int) -> np.ndarray:
    """Canonical representative of each string (backend/BAA.cu:216-227)."""
    xs = np.asarray(xs, dtype=np.uint64)
    m = np.uint64((1 << n) - 1)
    r = reverse_bits(xs, n)
    c = xs ^ m
    rc = reverse_bits(c, n)
    return np.minimum(np.minimum(xs, r), np.minimum(c, rc))


def orbit_average(full: np.ndarray, n: int) -> np.ndarray:
    """Per-representative mean of a vector over all 2^n strings."""
    full = np.asarray(full, dtype=np.float64)
    x = np.arange(1 << n, dtype=np.uint64)
    reps = canonical_reps(n).astype(np.uint64)
    idx = np.searchsorted(reps, rep_of(x, n))
    sums = np.bincount(idx, weights=full, minlength=len(reps))
    cnt = np.bincount(idx, minlength=len(reps)).astype(np.float64)
    return sums / cnt


def expand_to_full(p_rep: np.ndarray, n: int) -> np.ndarray:
    """Per-string vector over all 2^n strings from a per-representative one."""
    x = np.arange(1 << n, dtype=np.uint64)
    reps = canonical_reps(n).astype(np.uint64)
    return np.asarray(p_rep, dtype=np.float64)[np.searchsorted(reps, rep_of(x, n))]


def normalise(p_rep: np.ndarray, n: int, reps=None) -> np.ndarray:
    reps = canonical_reps(n) if reps is None else reps
    return p_rep / np.sum(orbit_sizes(reps, n) * p_rep)


def orbit_mean_at_reps(g: np.ndarray, n: int, reps=None) -> np.ndarray:
    """The same per-representative means as orbit_average, computed from the
    representatives' own orbits (O(#reps) work instead of O(2^n) searches):
    the distinct members of each orbit are added in ascending order, as
    orbit_average's bincount adds them, so the results agree bit for bit."""
    reps = (canonical_reps(n) if reps is None else reps).astype(np.uint64)
    m = np.uint64((1 << n) - 1)
    imgs = np.stack([reps, reverse_bits(reps, n), reps ^ m, reverse_bits(reps ^ m, n)], axis=1)
    imgs.sort(axis=1)
    g = np.asarray(g, dtype=np.float64)
    s = g[imgs[:, 0]].copy()
    cnt = np.ones(len(reps))
    for j in range(1, 4):
        new = imgs[:, j] != imgs[:, j - 1]
        s += np.where(new, g[imgs[:, j]], 0.0)
        cnt += new
    return s / cnt


def dirichlet_start(n: int, alpha: float, seed: int) -> np.ndarray:
    """Seeded Dirichlet(alpha) draw over all 2^n strings (normalised gamma
    variates from numpy's PCG64 generator), symmetrised by averaging over each
    orbit and stored per representative with sum |O| p = 1."""
    rng = np.random.default_rng(seed)
    g = rng.gamma(alpha, 1.0, size=1 << n)
    reps = canonical_reps(n)
    p = orbit_mean_at_reps(g, n, reps)
    return normalise(p, n, reps)


def uniform_start(n: int) -> np.ndarray:
    """p = 1 / 2^n per representative (backend/main_BAA.cu:64)."""
    return np.full(len(canonical_reps(n)), 1.0 / (1 << n))
