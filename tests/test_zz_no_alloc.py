"""The allocation-free entry point bdc_max_deviation_noalloc, through the C ABI.

It exists for callers that cannot allocate device memory (all of theirs comes
from their own pool or arena, or an allocator call is not allowed where they
run): they pass device buffers they own and the library uses a fixed scratch
array instead of allocating.  Checked against the allocating entry point
bdc_max_deviation on the same data, twice in a row (the shared scratch array
keeps the previous call's contents), with the same tolerance as the other
reductions (max is order-independent, so the results agree exactly).  This
file is collected last so a failure here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_max_deviation_matches_allocating_entry_point(bdc):
    import torch

    n, k = 16, 8
    with bdc.Engine(n, k, engine="count") as E:
        R = E.R
        rng = np.random.default_rng(2024)
        for call in range(2):
            p = rng.random(R) + 0.5
            pb = rng.random(R) + 0.5
            if call == 1:
                p[R // 3] *= 64.0  # a different maximum than the first call
            want = E.max_deviation(p, pb)
            tp = torch.tensor(p, dtype=torch.float64, device="cuda")
            tpb = torch.tensor(pb, dtype=torch.float64, device="cuda")
            out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
            stream = torch.cuda.current_stream().cuda_stream
            bdc.max_deviation_noalloc(tp.data_ptr(), tpb.data_ptr(), R, out.data_ptr(), stream)
            torch.cuda.synchronize()
            got = float(out.item())
            assert got == pytest.approx(want, rel=0, abs=1e-12), (call, got, want)
            assert got == pytest.approx(float(np.max(np.log2(p) - np.log2(pb))), abs=1e-12)


def test_noalloc_ragged_last_tile_and_many_partials(bdc):
    # 301 blocks of the fixed scratch, the last one holding 17 entries; the
    # maximum sits in that ragged tile on the first call and elsewhere on
    # the second, so a stale slot from the first call would show
    import torch

    R = 8192 * 300 + 17
    rng = np.random.default_rng(7)
    for call, where in enumerate((R - 5, 8192 * 150 + 3)):
        p = rng.random(R) + 0.5
        pb = rng.random(R) + 0.5
        p[where] *= 1024.0
        tp = torch.tensor(p, dtype=torch.float64, device="cuda")
        tpb = torch.tensor(pb, dtype=torch.float64, device="cuda")
        out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
        bdc.max_deviation_noalloc(tp.data_ptr(), tpb.data_ptr(), R, out.data_ptr(),
                                  torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        want = float(np.max(np.log2(p) - np.log2(pb)))
        assert float(out.item()) == pytest.approx(want, rel=0, abs=1e-12), (call, float(out.item()), want)


def test_noalloc_rejects_sizes_beyond_the_limit(bdc):
    L = bdc.library()
    rc = L.bdc_max_deviation_noalloc(ctypes.c_void_p(8), ctypes.c_void_p(8), (1 << 27) + 1,
                                     ctypes.c_void_p(8), None)
    assert rc == 1
    assert b"exceeds the fixed scratch limit" in L.bdc_last_error()
