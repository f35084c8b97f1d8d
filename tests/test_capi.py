"""The C ABI library: it loads, exports every function include/bdc_b200.h
declares, and its host-only parts (file formats, argument checks) behave
like the reference's (backend/cache_io.h, backend/main_BAA.cu:3-18) without
a GPU."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import GOLDEN, REPO


def header_functions():
    src = open(os.path.join(REPO, "include", "bdc_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bdc_[a-z_0-9]+)\s*\(", src)))


def test_library_exports_every_declared_function(bdc):
    L = bdc.library()
    declared = header_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(bdc.EXPORTED_SYMBOLS) == declared


def test_version_and_default_options(bdc):
    L = bdc.library()
    assert b"sm_100a" in L.bdc_version()
    o = bdc.Options()
    L.bdc_default_options(ctypes.byref(o))
    assert o.engine == 0 and o.device == 0 and o.cache_dir is None


def test_cache_file_roundtrip_and_reference_files(bdc, tmp_path, O):
    d = os.path.join(GOLDEN, "ref_caches")
    ref = bdc.read_cache_file(os.path.join(d, "cache_6_3"), 6, 3)
    assert np.array_equal(ref, O.gen_cache(6, 3))
    p = str(tmp_path / "cache_6_3")
    bdc.write_cache_file(p, 6, 3, ref)
    assert open(p, "rb").read() == open(os.path.join(d, "cache_6_3"), "rb").read()


def test_cache_file_size_checked(bdc, tmp_path):
    p = tmp_path / "cache_5_2"
    np.arange(10, dtype="<u4").tofile(p)
    with pytest.raises(bdc.BDCError) as e:
        bdc.read_cache_file(str(p), 5, 2)
    assert e.value.status == 3
    with pytest.raises(bdc.BDCError) as e:
        bdc.read_cache_file(str(tmp_path / "missing"), 5, 2)
    assert e.value.status == 3 and "failed to open file" in str(e.value)


def test_dist_file_roundtrip_is_exact(bdc, tmp_path):
    rng = np.random.default_rng(1)
    p = rng.random(1000) ** 7
    p[5] = 0.0
    f = str(tmp_path / "dist_10_5.txt")
    bdc.write_dist_file(f, p)
    lines = open(f).read().split("\n")
    assert lines[0] == "%.17g" % p[0] and lines[5] == "0"
    assert np.array_equal(bdc.read_dist_file(f), p)
    assert not os.path.exists(f + ".tmp")


def test_dist_file_errors(bdc, tmp_path):
    with pytest.raises(bdc.BDCError) as e:
        bdc.read_dist_file(str(tmp_path / "none.txt"))
    assert e.value.status == 3
    f = tmp_path / "bad.txt"
    f.write_text("0.5\n0.25\nabc\n")
    with pytest.raises(bdc.BDCError):
        bdc.read_dist_file(str(f))


def test_create_argument_checks(bdc):
    for n, k in [(0, 0), (5, 6), (31, 4), (12, 0)]:
        with pytest.raises(bdc.BDCError) as e:
            bdc.Engine(n, k)
        assert e.value.status == 1


def test_reference_shaped_calls_need_load_cache(bdc):
    with pytest.raises(bdc.BDCError):
        bdc.baa_iteration(np.ones(4), None, 4, 2)


def test_host_helpers_match_oracle(bdc, O):
    from bdc_b200 import dist
    for n in (5, 8, 11):
        assert np.array_equal(bdc.canonical_reps(n), O.canonicals(n))
        reps = O.canonicals(n)
        assert np.array_equal(bdc.orbit_sizes(reps, n), O.orbits_of(reps, n))
    p = dist.dirichlet_start(10, 1.0, 0)
    reps = O.canonicals(10)
    assert abs(np.sum(O.orbits_of(reps, 10) * p) - 1) < 1e-14
    full = dist.expand_to_full(p, 10)
    assert np.allclose(dist.orbit_average(full, 10), p, rtol=0, atol=0)


def test_orbit_means_from_representatives_are_bit_identical():
    # the O(#reps) orbit means (dist.orbit_mean_at_reps) against the O(2^n)
    # bincount over all strings (dist.orbit_average), odd and even n
    from bdc_b200 import dist
    for n in (7, 10, 13, 16):
        g = np.random.default_rng(n).gamma(0.5, 1.0, size=1 << n)
        assert np.array_equal(dist.orbit_mean_at_reps(g, n), dist.orbit_average(g, n))


def test_bit_reversal_table_matches_bitwise_definition(bdc):
    rng = np.random.default_rng(3)
    for n in (1, 5, 8, 12, 17, 24, 31):
        xs = rng.integers(0, 1 << n, 2000, dtype=np.uint64)
        want = np.array([int(format(int(x), f"0{n}b")[::-1], 2) for x in xs], dtype=np.uint64)
        assert np.array_equal(bdc.reverse_bits(xs, n).astype(np.uint64), want)


def test_dirichlet_starts_are_seeded():
    from bdc_b200 import dist
    a, b, c = dist.dirichlet_start(12, 0.5, 4), dist.dirichlet_start(12, 0.5, 4), dist.dirichlet_start(12, 0.5, 5)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert np.all(a > 0)
