"""The certified solver: its bracket is evaluated exactly at the point it
returns (checked with the oracle), it contains the plain BA's limit, and it
is below the requested gap."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LN2 = np.log(2.0)


def _bracket_at(O, n, k, p):
    reps = O.canonicals(n)
    lnq = O.log_q(n, k, p, reps)
    D = O.kl(n, k, lnq, reps)
    return O.rate(n, k, lnq, p, reps) / LN2, D.max() / LN2


@pytest.mark.parametrize("n,k,start", [(12, 6, None), (13, 7, ("dirichlet", 1.0, 1)), (16, 8, ("dirichlet", 0.5, 0))])
def test_solve_certifies_a_tight_bracket(bdc, O, n, k, start):
    from bdc_b200 import dist
    with bdc.Engine(n, k, engine="factored") as E:
        if start is None:
            E.set_uniform()
        else:
            E.set_p(dist.dirichlet_start(n, start[1], start[2]))
        st = E.solve(1e-9, 20000)
        assert st["converged"], st
        assert 0.0 <= st["best_upper_bound"] - st["best_rate"] < 1e-9
        # the returned point carries the certified numbers (oracle, CPU)
        p = E.get_p()
        reps = O.canonicals(n)
        assert abs(np.sum(O.orbits_of(reps, n) * p) - 1.0) < 1e-12
        rate, ub = _bracket_at(O, n, k, p)
        assert abs(rate - st["rate"]) < 1e-11
        assert abs(ub - st["upper_bound"]) < 1e-11
        assert st["best_rate"] <= ub + 1e-12 and rate <= st["best_upper_bound"] + 1e-12
        # the plain BA bracket after many iterations overlaps it (both hold C)
        E2 = bdc.Engine(n, k, engine="factored")
        E2.set_uniform()
        pl = E2.iterate(4000, float("-inf"))
        E2.close()
        assert pl["best_rate"] <= st["best_upper_bound"] + 1e-12
        assert st["best_rate"] <= pl["best_upper_bound"] + 1e-12
        assert st["best_upper_bound"] <= pl["best_upper_bound"] + 1e-12


def test_solve_iterate_keeps_zeros(bdc, O):
    # after the solver, plain iterations keep the zero entries at zero
    n, k = 12, 6
    with bdc.Engine(n, k, engine="factored") as E:
        E.set_uniform()
        st = E.solve(1e-9, 20000)
        p0 = E.get_p()
        E.iterate(3, float("-inf"))
        p1 = E.get_p()
        assert np.all(p1[p0 == 0.0] == 0.0)
        assert (p0 == 0.0).sum() > 0


def test_solve_errors(bdc):
    with bdc.Engine(8, 4, engine="count") as E:
        E.set_uniform()
        with pytest.raises(bdc.BDCError):
            E.solve(1e-9, 100)
    with bdc.Engine(8, 4, engine="factored") as E:
        with pytest.raises(bdc.BDCError):
            E.solve(1e-9, 100)   # no distribution
        E.set_uniform()
        with pytest.raises(bdc.BDCError):
            E.solve(0.0, 100)


def test_compute_c_n_k_plain_and_certified(bdc, O, tmp_path):
    # the reference-shaped driver (backend/main_BAA.cu:39-131): the plain loop
    # matches the oracle's; certified_gap gives a bracket holding its rate
    n, k = 10, 5
    plain = bdc.compute_C_n_k(n, k, a=1e-3, base=str(tmp_path), cache_dir=None, verbose=False)
    reps = O.canonicals(n)
    ref = O.run_ba(n, k, np.full(len(reps), 1.0 / (1 << n)), reps, 1e-3, 100000)
    assert plain["iters"] == ref["iters"]
    assert abs(plain["rate_bits"] - ref["rate_bits"]) < 1e-11
    cert = bdc.compute_C_n_k(n, k, base=str(tmp_path), cache_dir=None, verbose=False, certified_gap=1e-9)
    assert cert["converged"] and 0.0 <= cert["upper_bits"] - cert["lower_bits"] < 1e-9
    assert cert["lower_bits"] >= plain["rate_bits"] - 1e-12   # BA's rate never exceeds C
    assert os.path.exists(os.path.join(str(tmp_path), "distributions", f"dist_{n}_{k}.txt"))
