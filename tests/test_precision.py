"""The compensated-FP32 engine ("count-fp32c"): the count path with its q and
D sums in two-float FP32 accumulators.  Its iterates follow the oracle's FP64
iterates, and each reported bound comes with its error against an FP64
re-evaluation at the same iterate (bdc_bound_error), which must stay far
below the 1e-9-bit tolerance."""
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import PKG

pytestmark = pytest.mark.gpu

TOL_BITS = 1e-9


def _start(n, spec):
    from bdc_b200 import dist
    if spec is None:
        return dist.uniform_start(n)
    return dist.dirichlet_start(n, spec[0], spec[1])


@pytest.mark.parametrize("n,k,start", [(10, 5, None), (12, 6, None), (13, 7, (1.0, 0)), (16, 8, (0.5, 1))])
def test_fp32c_iterates_follow_the_fp64_oracle(bdc, O, n, k, start):
    iters, a = 12, 1e-30
    reps = O.canonicals(n)
    p0 = _start(n, start)
    ref = O.run_ba(n, k, p0, reps, a, iters)
    with bdc.Engine(n, k, engine="count-fp32c") as E:
        assert E.engine == "count-fp32c"
        E.set_p(p0)
        st = E.iterate(iters, a)
        assert st["iters"] == iters
        np.testing.assert_allclose(E.get_p(), ref["p"], rtol=1e-10, atol=1e-300)
        assert abs(st["mx"] - ref["mx_final"]) < 1e-9
        ub_err, rate_err = E.bound_error()
        assert 0.0 <= ub_err < 1e-11 and 0.0 <= rate_err < 1e-11
        # the FP64 count engine on the same iterates: the bound within the tolerance
        with bdc.Engine(n, k, engine="count") as F:
            F.set_p(p0)
            s64 = F.iterate(iters, a)
            assert F.bound_error() == (0.0, 0.0)
        assert abs(st["upper_bound"] - s64["upper_bound"]) < TOL_BITS
        assert abs(st["rate"] - s64["rate"]) < TOL_BITS


def test_fp32c_q_and_d_against_the_oracle(bdc, O):
    # one evaluation: ln q (the C ABI's compute_all_log_D) and D per representative
    n, k = 14, 7
    reps = O.canonicals(n)
    p = _start(n, (0.5, 3))
    with bdc.Engine(n, k, engine="count-fp32c") as E:
        E.set_p(p)
        lnq = E.log_q()
        d = E.divergence()
    lnq_ref = O.log_q(n, k, p, reps)
    d_ref = O.kl(n, k, lnq_ref, reps)
    np.testing.assert_allclose(lnq, lnq_ref, rtol=0, atol=1e-12)
    np.testing.assert_allclose(d, d_ref, rtol=0, atol=1e-12)


def test_fp32c_limits_and_state(bdc):
    with pytest.raises(bdc.BDCError):
        bdc.Engine(27, 13, engine="count-fp32c")      # counts above 2^24
    with bdc.Engine(9, 4, engine="count-fp32c") as E:
        E.set_uniform()
        with pytest.raises(bdc.BDCError):
            E.bound_error()                             # no iteration yet
        E.iterate(1, float("-inf"))
        assert E.bound_error()[0] >= 0.0


def test_fp32c_in_a_batch_matches_single_engines(bdc):
    mix = [(10, 5), (12, 6), (11, 3)]
    engines = [bdc.Engine(n, k, engine="count-fp32c") for n, k in mix]
    try:
        for E in engines:
            E.set_uniform()
        with bdc.Batch(engines) as B:
            stats = B.iterate(11, 1e-30)
        for E, st, (n, k) in zip(engines, stats, mix):
            with bdc.Engine(n, k, engine="count-fp32c") as S:
                S.set_uniform()
                s1 = S.iterate(11, 1e-30)
                np.testing.assert_array_equal(S.get_p(), E.get_p())
                assert s1["upper_bound"] == st["upper_bound"]
    finally:
        for E in engines:
            E.close()


def test_main_baa_fp32c_prints_its_bound_error(tmp_path, O):
    n, k, a = 12, 6, 1e-3
    d = tmp_path / "c32"
    (d / "distributions").mkdir(parents=True)
    env = dict(os.environ, BDC_TABLES="device", BDC_ENGINE="count-fp32c")
    r = subprocess.run([os.path.join(PKG, "main_BAA"), str(n), str(k), "0", str(a), "1000"], cwd=d, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    reps = O.canonicals(n)
    ref = O.run_ba(n, k, np.full(len(reps), 1.0 / (1 << n)), reps, a, 100000)
    line = f"Computed C_{{{n},{k}}} = {ref['rate_bits']:.6f} bits (max deviation {ref['mx_final']:.6f})"
    assert line in r.stdout.splitlines()
    m = re.search(r"^Compensated FP32: last bound (\S+) bits and rate (\S+) bits from their FP64 values$",
                  r.stdout, re.M)
    assert m, r.stdout
    assert float(m.group(1)) < 1e-11 and float(m.group(2)) < 1e-11
