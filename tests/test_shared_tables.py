"""Handles of one (n, k) on one device share their p-independent data.

The representatives, the half-table bundles, the rotated A bundle and h(x)
per representative are built by the first handle of an (n, k, table source)
and shared by every later one (the seeds of a batch): a second handle takes
far less device memory, iterates identically, and keeps working after the
first one is closed.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_second_handle_shares_tables(bdc):
    import torch
    n, k = 24, 12
    R = 4_196_352
    # reps, h, the bundle (one for both halves at even n) and its rotated copy
    tables = R * (4 + 8) + 2 * (4096 * 4096 * 2)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    E1 = bdc.Engine(n, k, engine="count")
    free1 = torch.cuda.mem_get_info()[0]
    E2 = bdc.Engine(n, k, engine="count")
    free2 = torch.cuda.mem_get_info()[0]
    first, second = free0 - free1, free1 - free2
    assert second < first - 0.9 * tables, (first, second, tables)
    rng = np.random.default_rng(3)
    p = rng.random(R)
    p /= p.sum()
    E1.set_p(p)
    E2.set_p(p)
    s1 = E1.iterate(2, float("-inf"))
    s2 = E2.iterate(2, float("-inf"))
    assert np.array_equal(E1.get_p(), E2.get_p())
    assert s1["upper_bound"] == s2["upper_bound"]
    p2 = E2.get_p()
    E1.close()
    # the tables outlive the handle that built them
    s3 = E2.iterate(1, float("-inf"))
    with bdc.Engine(n, k, engine="count") as E3:
        E3.set_p(p2)
        s4 = E3.iterate(1, float("-inf"))
        assert np.array_equal(E2.get_p(), E3.get_p())
        assert s3["upper_bound"] == s4["upper_bound"]
    E2.close()
    # all closed: a new handle builds the set again
    with bdc.Engine(12, 6, engine="count") as E4:
        E4.set_uniform()
        assert E4.iterate(3, float("-inf"))["iters"] == 3
