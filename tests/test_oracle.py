"""The CPU oracle against the reference's own outputs and known answers.

Pins: the reference cache generator's files (sha256 of every cache_n_k with
n <= 11, and small files verbatim, made by tests/golden/make_golden.py from
backend/generate_bit_transition_cache.cpp compiled unchanged); the analytic
capacities C_{n,1} = 1 and C_{n,n} = n (Upper_Bounds.txt:6,34,71-72); exact
identities of the channel (sum_y W = 1, symmetry invariance).
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN


def test_reference_cache_hashes(O):
    ref = json.load(open(os.path.join(GOLDEN, "ref_cache_sha256.json")))["sha256"]
    assert len(ref) == 66
    for name, digest in ref.items():
        _, n, k = name.split("_")
        n, k = int(n), int(k)
        mine = O.gen_cache(n, k).astype("<u4").tobytes()
        assert hashlib.sha256(mine).hexdigest() == digest, name


def test_reference_small_caches_verbatim(O):
    d = os.path.join(GOLDEN, "ref_caches")
    for f in sorted(os.listdir(d)):
        _, n, k = f.split("_")
        ref = np.fromfile(os.path.join(d, f), dtype="<u4")
        assert np.array_equal(ref, O.gen_cache(int(n), int(k))), f
    # spot values: row x=000 of cache_3_2 is [3,0,0,0]; row x=0000 of cache_4_2 is [6,0,0,0]
    assert list(np.fromfile(os.path.join(d, "cache_3_2"), dtype="<u4")[:4]) == [3, 0, 0, 0]
    assert list(np.fromfile(os.path.join(d, "cache_4_2"), dtype="<u4")[:4]) == [6, 0, 0, 0]


@pytest.mark.parametrize("n,k", [(12, 6), (13, 5), (9, 9), (9, 1), (20, 10), (24, 12), (26, 13), (7, 3)])
def test_split_identity_matches_dp(O, n, k):
    rng = np.random.default_rng(n * 100 + k)
    xs = rng.integers(0, 1 << n, 300)
    ys = rng.integers(0, 1 << k, 300)
    for x, y in zip(xs, ys):
        assert O.total_transitions(int(x), int(y), n, k) == O.count_dp(int(x), n, int(y), k)


@pytest.mark.parametrize("n,k", [(8, 4), (11, 5), (12, 6)])
def test_rows_sum_to_binomial(O, n, k):
    xs = np.arange(0, 1 << n, 37, dtype=np.uint32)
    rows = O.count_rows(n, k, xs)
    assert np.all(rows.sum(axis=1) == O.nck(n, k))  # sum_y W(y|x) = 1 exactly


def test_counts_symmetry_invariant(O):
    n, k = 11, 5
    rng = np.random.default_rng(5)
    for _ in range(200):
        x, y = int(rng.integers(1 << n)), int(rng.integers(1 << k))
        N = O.count_dp(x, n, y, k)
        rx = int(format(x, f"0{n}b")[::-1], 2)
        ry = int(format(y, f"0{k}b")[::-1], 2)
        cx, cy = x ^ ((1 << n) - 1), y ^ ((1 << k) - 1)
        assert O.count_dp(rx, n, ry, k) == N
        assert O.count_dp(cx, n, cy, k) == N


@pytest.mark.parametrize("n", [4, 8, 12, 20])
def test_burnside_rep_count(O, n):
    expect = ((1 << n) + (1 << ((n + 1) // 2)) + ((1 << (n // 2)) if n % 2 == 0 else 0)) // 4
    assert len(O.canonicals(n)) == expect


def test_distinct_subsequences_are_the_support(O):
    n, k = 10, 4
    for x in (0, 1, 0b1010101010, 0b1100110011, 777):
        ys = set(int(v) for v in O.distinct_subsequences(x, n, k))
        support = {y for y in range(1 << k) if O.count_dp(x, n, y, k) > 0}
        assert ys == support


@pytest.mark.parametrize("n", [5, 8])
def test_known_capacity_k1_and_kn(O, n):
    reps = O.canonicals(n)
    p = np.full(len(reps), 1.0 / (1 << n))
    r1 = O.run_ba(n, 1, p, reps, 1e-9, 5000)
    assert abs(r1["rate_bits"] - 1.0) < 1e-8
    rn = O.run_ba(n, n, p, reps, 1e-9, 10)
    assert abs(rn["rate_bits"] - n) < 1e-12
    assert rn["iters"] == 1  # uniform is already optimal: mx = 0 < a after one step


def test_iterate_stays_normalised_and_bounds_bracket(O):
    n, k = 10, 5
    reps = O.canonicals(n)
    orb = O.orbits_of(reps, n)
    p = np.full(len(reps), 1.0 / (1 << n))
    prev_rate = -1.0
    for t in range(8):
        pn, lnq, lw = O.ba_iteration(n, k, p, reps)
        assert abs(np.sum(orb * pn) - 1.0) < 1e-13
        d = lw - np.log(p)
        ub = d.max() / np.log(2)
        rate = np.sum(orb * p * d) / np.log(2)
        assert rate <= ub + 1e-12
        assert rate >= prev_rate - 1e-12      # BA rate is non-decreasing
        prev_rate = rate
        p = pn


def test_zero_entries_follow_reference_log_rule(O):
    # ln 0 is taken as 0 (backend/BAA.cu:573-580): a zero p(x) re-enters
    # with weight e^{D(x)} after one step
    n, k = 8, 4
    reps = O.canonicals(n)
    p = np.full(len(reps), 1.0 / (1 << n))
    p[3] = 0.0
    pn, lnq, lw = O.ba_iteration(n, k, p, reps)
    assert pn[3] > 0
    assert O.max_deviation(pn, p) == np.inf
