"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Counts are compared bit-exactly; ln q, ln p + D, D and p' within the
tolerances below (FP64 sums in a different order than the reference's):
  TOL_REL = 1e-12 relative on q and p', TOL_ABS = 1e-12 absolute on ln q,
  logW and D (all O(1..20) in size).
The compensated-FP32 engine (count-fp32c) is held to the same tolerances in
the single-pass and iterate checks.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TOL_REL = 1e-12
TOL_ABS = 1e-12

ENGINES = ["count", "factored"]
NUMERIC_ENGINES = ENGINES + ["count-fp32c"]


def start(n, kind, O):
    from bdc_b200 import dist
    if kind == "uniform":
        return np.full(len(O.canonicals(n)), 1.0 / (1 << n))
    if kind == "dirichlet":
        return dist.dirichlet_start(n, 1.0, 0)
    if kind == "zeros":
        p = dist.dirichlet_start(n, 1.0, 7)
        p[::5] = 0.0
        return p
    raise ValueError(kind)


def test_generated_caches_match_reference_generator(bdc):
    ref = json.load(open(os.path.join(GOLDEN, "ref_cache_sha256.json")))["sha256"]
    for name, digest in ref.items():
        _, n, k = name.split("_")
        out = bdc.generate_cache(int(n), int(k))
        assert hashlib.sha256(out.astype("<u4").tobytes()).hexdigest() == digest, name


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("n,k", [(12, 6), (13, 5), (20, 10), (24, 12), (9, 9), (9, 1), (7, 3), (16, 10)])
def test_reps_and_counts_bit_exact(bdc, O, engine, n, k):
    if engine == "factored" and k >= n:
        pytest.skip("the factored engine needs k < n")
    with bdc.Engine(n, k, engine=engine) as E:
        if n <= 20:
            assert np.array_equal(E.reps, O.canonicals(n))
        else:
            assert len(E.reps) == ((1 << n) + (1 << ((n + 1) // 2)) + (1 << (n // 2))) // 4
            assert np.all(np.diff(E.reps.astype(np.int64)) > 0)
        rng = np.random.default_rng(n * 31 + k)
        xs = rng.integers(0, 1 << n, 4000).astype(np.uint32)
        ys = rng.integers(0, 1 << k, 4000).astype(np.uint32)
        # include subsequences of x so most counts are non-zero
        for i in range(0, 4000, 2):
            pos = np.sort(rng.choice(n, k, replace=False))
            bits = [(int(xs[i]) >> (n - 1 - q)) & 1 for q in pos]
            ys[i] = int("".join(map(str, bits)), 2)
        got = E.counts(xs, ys)
        want = np.array([O.count_dp(int(x), n, int(y), k) for x, y in zip(xs, ys)], dtype=np.uint32)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("engine", NUMERIC_ENGINES)
@pytest.mark.parametrize("n,k,kind", [(12, 6, "uniform"), (13, 5, "uniform"), (10, 4, "dirichlet"),
                                      (16, 8, "dirichlet"), (10, 5, "zeros"), (9, 9, "uniform"),
                                      (9, 1, "dirichlet"), (11, 10, "dirichlet"), (14, 3, "dirichlet")])
def test_single_passes_match_oracle(bdc, O, engine, n, k, kind):
    if engine == "factored" and k >= n:
        pytest.skip("the factored engine needs k < n")
    reps = O.canonicals(n)
    p = start(n, kind, O)
    with bdc.Engine(n, k, engine=engine) as E:
        E.set_p(p)
        lnq = E.log_q()
        lnq_o = O.log_q(n, k, p, reps)
        np.testing.assert_allclose(lnq, lnq_o, rtol=0, atol=TOL_ABS)
        lw = E.log_w()
        np.testing.assert_allclose(lw, O.log_w(n, k, p, lnq_o, reps), rtol=0, atol=TOL_ABS * 10)
        d = E.divergence(lnq_o)
        np.testing.assert_allclose(d, O.kl(n, k, lnq_o, reps), rtol=0, atol=TOL_ABS)
        r = E.rate()
        assert abs(r - O.rate(n, k, lnq_o, p, reps)) < 1e-12
        pn = E.baa_iteration(p)
        pn_o, _, _ = O.ba_iteration(n, k, p, reps)
        np.testing.assert_allclose(pn, pn_o, rtol=TOL_REL, atol=0)


@pytest.mark.parametrize("engine", NUMERIC_ENGINES)
@pytest.mark.parametrize("n,k,kind,iters", [(12, 6, "uniform", 25), (13, 7, "dirichlet", 10),
                                            (16, 8, "dirichlet", 5)])
def test_iterates_track_oracle(bdc, O, engine, n, k, kind, iters):
    reps = O.canonicals(n)
    p0 = start(n, kind, O)
    ref = O.run_ba(n, k, p0, reps, -1.0, iters)   # a < 0: never stops early
    with bdc.Engine(n, k, engine=engine) as E:
        E.set_p(p0)
        st = E.iterate(iters, -1.0)
        assert st["iters"] == iters and not st["converged"]
        np.testing.assert_allclose(E.get_p(), ref["p"], rtol=1e-11, atol=0)
        assert abs(st["mx"] - ref["mx"][-1]) < 1e-11
        assert abs(st["upper_bound"] - ref["ub_bits"][-1]) < 1e-11


@pytest.mark.parametrize("engine", ENGINES)
def test_stopping_rule_matches_reference_loop(bdc, O, engine):
    n, k, a = 12, 6, 1e-5
    reps = O.canonicals(n)
    p0 = start(n, "uniform", O)
    ref = O.run_ba(n, k, p0, reps, a, 100000)
    with bdc.Engine(n, k, engine=engine) as E:
        E.set_p(p0)
        st = E.iterate(100000, a)
        assert st["converged"]
        assert st["iters"] == ref["iters"]
        assert abs(st["mx"] - ref["mx_final"]) < 1e-12
        # after thousands of iterations the smallest probabilities (< 1e-150,
        # down to denormals) carry the accumulated rounding of their logs
        p, pr = E.get_p(), ref["p"]
        big = pr > 1e-150
        np.testing.assert_allclose(p[big], pr[big], rtol=1e-10, atol=0)
        assert np.all(np.abs(p[~big] - pr[~big]) < 1e-150)
        assert abs(E.rate() / np.log(2) - ref["rate_bits"]) < 1e-11


def test_cache_dir_tables_equal_generated(bdc, O, tmp_path):
    n, k = 12, 6
    d = tmp_path / "transition_counts"
    d.mkdir()
    for m in range(0, 6):
        bdc.write_cache_file(str(d / f"cache_6_{m}"), 6, m, O.gen_cache(6, m))
    p = start(n, "dirichlet", O) if False else np.full(len(O.canonicals(n)), 1.0 / (1 << n))
    with bdc.Engine(n, k, engine="count", cache_dir=str(d)) as E1, bdc.Engine(n, k, engine="count") as E2:
        E1.set_p(p)
        E2.set_p(p)
        assert np.array_equal(E1.log_q(), E2.log_q())
    (d / "cache_6_3").unlink()
    with pytest.raises(bdc.BDCError) as e:
        bdc.Engine(n, k, engine="count", cache_dir=str(d))
    assert e.value.status == 3


def test_argument_errors_on_device(bdc, O):
    with bdc.Engine(10, 5, engine="count") as E:
        with pytest.raises(bdc.BDCError) as e:
            E.set_p(np.ones(E.R + 1))
        assert e.value.status == 1
        with pytest.raises(bdc.BDCError) as e:
            E.get_p()
        assert e.value.status == 5
        with pytest.raises(bdc.BDCError) as e:
            E.counts([1 << 10], [0])
        assert e.value.status == 1


def test_reference_shaped_api(bdc, O):
    n, k = 11, 5
    reps = O.canonicals(n)
    p = start(n, "uniform", O)
    bdc.load_cache(n, k, cache_dir=None)
    lnq = bdc.compute_all_log_D(p, reps, n, k)
    np.testing.assert_allclose(lnq, O.log_q(n, k, p, reps), rtol=0, atol=TOL_ABS)
    lw = bdc.compute_all_log_W(p, lnq, reps, n, k)
    np.testing.assert_allclose(lw, O.log_w(n, k, p, lnq, reps), rtol=0, atol=1e-11)
    pn = bdc.baa_iteration(p, reps, n, k)
    np.testing.assert_allclose(pn, O.ba_iteration(n, k, p, reps)[0], rtol=TOL_REL, atol=0)
    assert abs(bdc.compute_rate(lnq, p, reps, n, k) - O.rate(n, k, lnq, p, reps)) < 1e-12
    assert bdc.compute_max_deviation(pn, p) == pytest.approx(O.max_deviation(pn, p), abs=1e-13)


@pytest.mark.parametrize("n,k", [(14, 7), (15, 6), (17, 9), (18, 6), (12, 11), (11, 2), (16, 14), (19, 14)])
def test_factored_equals_count_engine(bdc, O, n, k):
    """The two engines run the same iteration: after 6 iterations from a
    Dirichlet start their iterates and statistics agree to rounding."""
    from bdc_b200 import dist
    p0 = dist.dirichlet_start(n, 0.5, 11)
    out = {}
    for engine in ("count", "factored"):
        with bdc.Engine(n, k, engine=engine) as E:
            assert E.engine == engine
            E.set_p(p0)
            st = E.iterate(6, -1.0)
            out[engine] = (E.get_p(), st)
    (pc, sc), (pf, sf) = out["count"], out["factored"]
    np.testing.assert_allclose(pf, pc, rtol=1e-11, atol=0)
    for key in ("mx", "upper_bound", "rate", "lse"):
        assert abs(sf[key] - sc[key]) < 1e-11, key
    assert sf["iters"] == sc["iters"] == 6


def test_factored_rescales_extreme_start(bdc, O):
    """An unnormalised start scaled by 1e-280 (the reference does not
    renormalise its input) puts exp(logW - shift) far out of range in the
    first fused update; the engine re-scales and still matches the oracle."""
    from bdc_b200 import dist
    n, k = 12, 6
    reps = O.canonicals(n)
    p0 = dist.dirichlet_start(n, 1.0, 5) * 1e-280
    ref = O.run_ba(n, k, p0, reps, -1.0, 3)
    with bdc.Engine(n, k, engine="factored") as E:
        E.set_p(p0)
        st = E.iterate(3, -1.0)
        assert st["iters"] == 3
        np.testing.assert_allclose(E.get_p(), ref["p"], rtol=1e-11, atol=0)
        assert abs(st["upper_bound"] - ref["ub_bits"][-1]) < 1e-11
        assert abs(st["mx"] - ref["mx"][-1]) < 1e-11


def test_underflowed_entries_reenter_like_reference(bdc, O):
    """Entries that are exactly 0 take ln p = 0 (backend/BAA.cu:573-580) in
    every iteration, in both engines, as in the oracle."""
    from bdc_b200 import dist
    n, k = 10, 5
    reps = O.canonicals(n)
    p0 = dist.dirichlet_start(n, 1.0, 9)
    p0[::7] = 0.0
    ref = O.run_ba(n, k, p0, reps, -1.0, 4)
    for engine in ("count", "factored"):
        with bdc.Engine(n, k, engine=engine) as E:
            E.set_p(p0)
            st = E.iterate(1, -1.0)
            assert np.isinf(st["mx"])
            st = E.iterate(3, -1.0)
            np.testing.assert_allclose(E.get_p(), ref["p"], rtol=1e-11, atol=0)


def test_engine_selection_by_size(bdc):
    # k = n has no factored form (W is the identity): auto takes the count path
    with bdc.Engine(12, 12) as E:
        assert E.engine == "count"
    with pytest.raises(bdc.BDCError) as e:
        bdc.Engine(12, 12, engine="factored")
    assert e.value.status == 6
    with bdc.Engine(16, 14) as E:
        assert E.engine == "factored"
