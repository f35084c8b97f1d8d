"""The adjoint of I(p;W) and the accelerated BA loop (forms beyond the
reference's plain loop): the gradient against central finite differences and against
the oracle's D(x); the accelerated loop against plain BA."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("engine", ["count", "factored"])
def test_adjoint_matches_finite_differences_and_oracle(bdc, O, engine):
    from bdc_b200 import dist
    n, k = 12, 6
    reps = O.canonicals(n)
    p0 = dist.dirichlet_start(n, 1.0, 3)
    with bdc.Engine(n, k, engine=engine) as E:
        I0 = E.mi_forward(p0)
        lnq = O.log_q(n, k, p0, reps)
        assert abs(I0 - O.rate(n, k, lnq, p0, reps)) < 1e-12
        g = E.mi_backward()
        # the closed form |O| (D - 1) with the oracle's D (backend/BAA.cu:413-425)
        np.testing.assert_allclose(g, O.orbits_of(reps, n) * (O.kl(n, k, lnq, reps) - 1.0), rtol=0, atol=1e-11)
        # central finite differences, h = 1e-7, on 64 seeded coordinates
        rng = np.random.default_rng(0)
        h = 1e-7
        for i in rng.choice(len(reps), 64, replace=False):
            pp, pm = p0.copy(), p0.copy()
            pp[i] += h
            pm[i] -= h
            fd = (E.mi_forward(pp) - E.mi_forward(pm)) / (2 * h)
            assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_device_backward_matches_the_host_backward(bdc, O):
    # the device-pointer form of the adjoint, for optimisers that keep the
    # iterate on the GPU: set_p_device -> mi_forward(None) -> mi_backward_device
    import torch
    from bdc_b200 import dist
    n, k = 12, 6
    reps = O.canonicals(n)
    p0 = dist.dirichlet_start(n, 1.0, 5)
    with bdc.Engine(n, k, engine="factored") as E:
        tp = torch.tensor(p0, dtype=torch.float64, device="cuda")
        E.set_p_device(tp.data_ptr())
        I0 = E.mi_forward(None)
        g = torch.empty_like(tp)
        E.mi_backward_device(g.data_ptr())
        host = E.mi_backward()
        np.testing.assert_array_equal(g.cpu().numpy(), host)
        lnq = O.log_q(n, k, p0, reps)
        assert abs(I0 - O.rate(n, k, lnq, p0, reps)) < 1e-12
        np.testing.assert_allclose(host, O.orbits_of(reps, n) * (O.kl(n, k, lnq, reps) - 1.0), rtol=0, atol=1e-11)


def test_accelerated_reaches_the_plain_bound_in_fewer_evaluations(bdc, O):
    n, k, tol = 12, 6, 1e-9
    with bdc.Engine(n, k, engine="factored") as E:
        E.set_uniform()
        ref = E.iterate(60000, -1.0)
        C = ref["best_upper_bound"]           # the plain BA's converged bound
        assert C - ref["best_rate"] < 1e-9
        # plain BA: evaluations until the bound is within tol of C
        E.set_uniform()
        plain = 0
        while True:
            st = E.iterate(500, -1.0)
            plain += st["iters"]
            if st["best_upper_bound"] - C < tol:
                break
        # accelerated: same criterion
        E.set_uniform()
        acc = 0
        while True:
            st = E.accelerate(300, 0.0)
            acc += st["iters"]
            assert st["best_upper_bound"] >= st["best_rate"] - 1e-12   # still a valid bracket
            if st["best_upper_bound"] - C < tol:
                break
            assert acc < plain, "accelerated loop fell behind plain BA"
        assert st["best_upper_bound"] >= C - 1e-9   # an upper bound cannot go below C
        assert acc * 2 < plain, (acc, plain)


def test_accelerated_stops_on_the_certified_gap(bdc):
    with bdc.Engine(10, 5, engine="factored") as E:
        E.set_uniform()
        st = E.accelerate(200000, 1e-8)
        assert st["converged"] == 1
        assert 0 <= st["best_upper_bound"] - st["best_rate"] < 1e-8
        p = E.get_p()
        reps = E.reps
        assert abs(np.sum(bdc.orbit_sizes(reps, 10) * p) - 1.0) < 1e-12
