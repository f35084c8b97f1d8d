"""The workloads the benchmark configurations name, under -m gpu.

* BDC_{20,10} from the Dirichlet(1) seed-0 start with the stopping threshold
  a = 1e-10 (the reference's loop, backend/main_BAA.cu:73-109): both FP64
  engines take the same iterates, the reference's rule does not stop them
  (mx stays above a), and at the final iterate ln q and D(x) agree with the
  CPU oracle to 1e-12 nats, counts bit-exact.  Plain BA cannot reach mx <
  1e-10 here in feasible time (mx = bound - log-sum-exp >= bound - C, and
  the bound was measured 7.4e-8 bits above C after 778,176 iterations), so
  the bound to that precision comes from the certified solver, whose
  bracket the oracle re-evaluates at the returned point.
* BDC_{26,13}: the adjoint dI/dp from the device backward against FP64
  central differences (h = 1e-7) on 1,024 seeded coordinates of a
  Dirichlet(1) start, and against the closed form |O| (D - 1) with the
  oracle's D on those coordinates (ln q from the count engine, an
  independent path, itself checked against the factored engine's).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LN2 = np.log(2.0)


def test_config2_20_10_dirichlet_seed0(bdc, O):
    from bdc_b200 import dist
    n, k, a, iters = 20, 10, 1e-10, 2000
    reps = O.canonicals(n)
    p0 = dist.dirichlet_start(n, 1.0, 0)
    with bdc.Engine(n, k, engine="factored") as F, bdc.Engine(n, k, engine="count") as Cn:
        # counts bit-exact against the oracle's split identity
        rng = np.random.default_rng(20)
        xs = rng.integers(0, 1 << n, 4096, dtype=np.uint32)
        ys = rng.integers(0, 1 << k, 4096, dtype=np.uint32)
        assert np.array_equal(F.counts(xs, ys), O.counts_pairs(n, k, xs, ys))
        F.set_p(p0)
        Cn.set_p(p0)
        sf = F.iterate(iters, a)
        sc = Cn.iterate(iters, a)
        # the reference's rule (while mx >= a) keeps going: neither engine stopped
        assert sf["iters"] == sc["iters"] == iters
        assert not sf["converged"] and not sc["converged"]
        assert sf["mx"] >= a and sc["mx"] >= a
        pf, pc = F.get_p(), Cn.get_p()
        np.testing.assert_allclose(pf, pc, rtol=1e-11, atol=0)
        # one more iteration against the oracle's own step from the same point
        lnq_o = O.log_q(n, k, pf, reps)
        kl_o = O.kl(n, k, lnq_o, reps)
        F.set_p(pf)
        np.testing.assert_allclose(F.log_q(), lnq_o, rtol=0, atol=1e-12)
        np.testing.assert_allclose(F.divergence(lnq_o), kl_o, rtol=0, atol=1e-12)
        pn_o, _, _ = O.ba_iteration(n, k, pf, reps)
        mx_o = O.max_deviation(pn_o, pf)
        s1 = F.iterate(1, a)
        np.testing.assert_allclose(F.get_p(), pn_o, rtol=1e-11, atol=0)
        assert abs(s1["mx"] - mx_o) < 1e-12
        assert abs(s1["upper_bound"] - kl_o.max() / LN2) < 1e-12
    # the bound to 1e-10 bits: the certified bracket from the same start,
    # re-evaluated by the oracle at the point the solver returns
    with bdc.Engine(n, k, engine="factored") as F:
        F.set_p(p0)
        st = F.solve(a, 200000)
        assert st["converged"] == 1
        lo, hi = st["best_rate"], st["best_upper_bound"]
        assert 0 <= hi - lo < a
        p = F.get_p()
        lnq = O.log_q(n, k, p, reps)
        rate_o = O.rate(n, k, lnq, p, reps) / LN2
        ub_o = O.kl(n, k, lnq, reps).max() / LN2
        assert abs(rate_o - st["rate"]) < 1e-12
        assert abs(ub_o - st["upper_bound"]) < 1e-12
        assert rate_o <= ub_o


def test_config5_26_13_adjoint_against_differences_and_closed_form(bdc, O):
    import torch
    from bdc_b200 import dist
    n, k, h, ncoord = 26, 13, 1e-7, 1024
    p0 = dist.dirichlet_start(n, 1.0, 0)
    with bdc.Engine(n, k, engine="factored") as E:
        reps = E.reps
        R = E.R
        tp = torch.tensor(p0, dtype=torch.float64, device="cuda")
        E.set_p_device(tp.data_ptr())
        I0 = E.mi_forward(None)
        g_dev = torch.empty_like(tp)
        E.mi_backward_device(g_dev.data_ptr())
        g = g_dev.cpu().numpy()
        lnq_f = E.log_q()
        rng = np.random.default_rng(0)
        idx = rng.choice(R, ncoord, replace=False)
        worst = 0.0
        for i in idx:
            i = int(i)
            v = float(p0[i])
            tp[i] = v + h
            E.set_p_device(tp.data_ptr())
            ip = E.mi_forward(None)
            tp[i] = v - h
            E.set_p_device(tp.data_ptr())
            im = E.mi_forward(None)
            tp[i] = v
            fd = (ip - im) / (2 * h)
            worst = max(worst, abs(fd - g[i]) / max(1.0, abs(g[i])))
        # rounding of I (~3 nats) over 2h bounds the differences' accuracy
        assert worst < 5e-8, worst
    with bdc.Engine(n, k, engine="count") as Cn:
        Cn.set_p(p0)
        lnq_c = Cn.log_q()
        assert abs(Cn.rate() - I0) < 1e-11
    np.testing.assert_allclose(lnq_f, lnq_c, rtol=0, atol=1e-12)
    sub = reps[idx]
    D_o = O.kl(n, k, lnq_c, sub)
    np.testing.assert_allclose(g[idx], O.orbits_of(sub, n) * (D_o - 1.0), rtol=0, atol=1e-11)
