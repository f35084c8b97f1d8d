"""Batches: several (n,k) instances and starting distributions iterated from
one captured CUDA graph must give, instance by instance, exactly what each
engine gives when iterated on its own, and the oracle's iterates."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (n, k, start): a mix of engines, sizes and starts, including one that stops early
MIX = [(10, 5, ("dirichlet", 0.5, 0)), (12, 6, ("uniform",)), (11, 3, ("dirichlet", 0.5, 1)),
       (9, 8, ("uniform",)), (13, 7, ("dirichlet", 1.0, 2))]


def _start(n, spec):
    from bdc_b200 import dist
    if spec[0] == "uniform":
        return dist.uniform_start(n)
    return dist.dirichlet_start(n, spec[1], spec[2])


@pytest.mark.parametrize("engine", ["count", "factored"])
def test_batch_matches_single_engines_and_oracle(bdc, O, engine):
    iters, a = 19, 1e-30          # 19 = two graph replays of 8 + 3 single steps
    engines = [bdc.Engine(n, k, engine=engine) for n, k, _ in MIX]
    try:
        for E, (n, k, spec) in zip(engines, MIX):
            E.set_p(_start(n, spec))
        with bdc.Batch(engines) as B:
            stats = B.iterate(iters, a)
        for E, st, (n, k, spec) in zip(engines, stats, MIX):
            reps = O.canonicals(n)
            ref = O.run_ba(n, k, _start(n, spec), reps, a, iters)
            assert st["iters"] == ref["iters"] == iters
            got = E.get_p()
            np.testing.assert_allclose(got, ref["p"], rtol=1e-10, atol=1e-300)
            assert abs(st["mx"] - ref["mx_final"]) < 1e-9
            # the same instance iterated alone
            with bdc.Engine(n, k, engine=engine) as S:
                S.set_p(_start(n, spec))
                s1 = S.iterate(iters, a)
                np.testing.assert_allclose(S.get_p(), got, rtol=1e-12, atol=1e-300)
                assert abs(s1["upper_bound"] - st["upper_bound"]) < 1e-12
    finally:
        for E in engines:
            E.close()


def test_batch_stops_each_instance_by_its_own_rule(bdc, O):
    # 9/8 converges in a few iterations; 12/6 does not: the first must stop at
    # the reference's own iteration count while the second runs on.
    a = 1e-6
    mix = [(9, 8), (12, 6)]
    engines = [bdc.Engine(n, k, engine="factored") for n, k in mix]
    try:
        for E in engines:
            E.set_uniform()
        with bdc.Batch(engines) as B:
            stats = B.iterate(200, a)
        for E, st, (n, k) in zip(engines, stats, mix):
            reps = O.canonicals(n)
            ref = O.run_ba(n, k, np.full(len(reps), 1.0 / (1 << n)), reps, a, 200)
            assert st["iters"] == ref["iters"], (n, k, st["iters"], ref["iters"])
            assert st["converged"] == (ref["iters"] < 200)
            np.testing.assert_allclose(E.get_p(), ref["p"], rtol=1e-10, atol=1e-300)
    finally:
        for E in engines:
            E.close()


def test_batch_argument_errors(bdc):
    with bdc.Engine(8, 4) as E:
        with pytest.raises(bdc.BDCError):
            bdc.Batch([E, E])
        with pytest.raises(bdc.BDCError):
            bdc.Batch([])
        with bdc.Batch([E]) as B:
            with pytest.raises(bdc.BDCError):
                B.iterate(4, 1e-9)     # no distribution set


def test_batch_accelerate_brackets_each_instance_and_times_it(bdc, O):
    # the accelerated loop of every instance from one graph, each stopping on
    # its own bracket; the bracket must hold in the oracle at the returned
    # point and match the same instance accelerated alone
    gap = 1e-9
    mix = [(10, 5, ("dirichlet", 0.5, 0)), (12, 6, ("uniform",)), (13, 6, ("dirichlet", 0.5, 1)),
           (14, 7, ("dirichlet", 1.0, 2))]
    engines = [bdc.Engine(n, k, engine="factored") for n, k, _ in mix]
    try:
        for E, (n, k, spec) in zip(engines, mix):
            E.set_p(_start(n, spec))
        with bdc.Batch(engines) as B:
            stats, secs = B.accelerate(200000, gap)
        for E, st, sec, (n, k, spec) in zip(engines, stats, secs, mix):
            assert st["converged"] == 1, (n, k, st)
            assert 0 <= st["best_upper_bound"] - st["best_rate"] < gap
            assert sec > 0
            with bdc.Engine(n, k, engine="factored") as S:
                S.set_p(_start(n, spec))
                s1 = S.accelerate(200000, gap)
            assert s1["converged"] == 1
            # two certified brackets of the same C overlap
            assert s1["best_rate"] <= st["best_upper_bound"] + 1e-12
            assert st["best_rate"] <= s1["best_upper_bound"] + 1e-12
            # the returned iterate is a distribution whose rate (oracle) is a
            # lower bound within the bracket's reach
            reps = O.canonicals(n)
            p = E.get_p()
            assert abs(np.sum(O.orbits_of(reps, n) * p) - 1.0) < 1e-12
            lnq = O.log_q(n, k, p, reps)
            rate_bits = O.rate(n, k, lnq, p, reps) / np.log(2.0)
            assert rate_bits <= st["best_upper_bound"] + 1e-12
    finally:
        for E in engines:
            E.close()
