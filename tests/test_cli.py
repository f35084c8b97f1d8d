"""The two command-line drop-ins against the reference programs built from the
reference sources (oracle/_ref/, when present) and against the oracle: same
argv, same files written, same result line."""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import PKG, REPO

pytestmark = pytest.mark.gpu

OUR_MAIN = os.path.join(PKG, "main_BAA")
OUR_GEN = os.path.join(PKG, "generate_bit_transition_cache")
REF_MAIN = os.path.join(REPO, "oracle", "_ref", "main_BAA")
REF_GEN = os.path.join(REPO, "oracle", "_ref", "generate_bit_transition_cache")


def _workdir(tmp_path, name, gen, max_n):
    d = tmp_path / name
    (d / "transition_counts").mkdir(parents=True)
    (d / "distributions").mkdir()
    subprocess.run([gen, str(max_n)], cwd=d, check=True, stdout=subprocess.DEVNULL, timeout=300)
    return d


def _run(exe, cwd, *argv):
    r = subprocess.run([exe, *map(str, argv)], cwd=cwd, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return r.stdout


def _summary(out):
    iters = [float(m) for m in re.findall(r"^Iteration \d+: mx = (\S+),", out, re.M)]
    res = re.search(r"^Computed C_\{(\d+),(\d+)\} = (\S+) bits \(max deviation (\S+)\)$", out, re.M)
    assert res, out
    return iters, res.group(0)


def _dist(d, n, k):
    return np.loadtxt(d / "distributions" / f"dist_{n}_{k}.txt")


def test_generator_writes_the_reference_files(tmp_path):
    if not os.path.exists(REF_GEN):
        pytest.skip("reference generator not built")
    ours = _workdir(tmp_path, "ours", OUR_GEN, 9)
    ref = _workdir(tmp_path, "ref", REF_GEN, 9)
    names = sorted(os.listdir(ref / "transition_counts"))
    assert names == sorted(os.listdir(ours / "transition_counts"))
    for f in names:
        a = (ours / "transition_counts" / f).read_bytes()
        b = (ref / "transition_counts" / f).read_bytes()
        assert a == b, f


@pytest.mark.parametrize("engine", ["count", "factored"])
def test_main_baa_matches_the_oracle_loop(tmp_path, O, engine, monkeypatch):
    n, k, a, save = 12, 6, 1e-3, 7
    monkeypatch.setenv("BDC_ENGINE", engine)
    ours = _workdir(tmp_path, "ours", OUR_GEN, (n + 1) // 2)
    out = _run(OUR_MAIN, ours, n, k, 0, a, save)
    it_ours, line_ours = _summary(out)
    p_ours = _dist(ours, n, k)
    # the oracle's outer loop (main_BAA.cu:39-131)
    reps = O.canonicals(n)
    ref = O.run_ba(n, k, np.full(len(reps), 1.0 / (1 << n)), reps, a, 100000)
    assert len(it_ours) == ref["iters"]
    np.testing.assert_allclose(it_ours, ref["mx"], rtol=0, atol=5e-7)   # printed with %.6f
    np.testing.assert_allclose(p_ours, ref["p"], rtol=1e-10, atol=0)
    assert line_ours == f"Computed C_{{{n},{k}}} = {ref['rate_bits']:.6f} bits (max deviation {ref['mx_final']:.6f})"


@pytest.mark.parametrize("engine", ["count", "factored"])
def test_main_baa_matches_the_reference_cli(tmp_path, engine, monkeypatch):
    # the reference's own main_BAA and generator, built unchanged from its
    # sources into oracle/_ref/ (oracle/Makefile ref)
    if not (os.path.exists(REF_MAIN) and os.path.exists(REF_GEN)):
        pytest.skip("the reference's main_BAA / generator are not built (oracle/Makefile ref)")
    n, k, a, save = 12, 6, 1e-3, 7
    monkeypatch.setenv("BDC_ENGINE", engine)
    ours = _workdir(tmp_path, "ours", OUR_GEN, (n + 1) // 2)
    it_ours, line_ours = _summary(_run(OUR_MAIN, ours, n, k, 0, a, save))
    refd = _workdir(tmp_path, "ref", REF_GEN, (n + 1) // 2)
    it_ref, line_ref = _summary(_run(REF_MAIN, refd, n, k, 0, a, save))
    assert line_ours == line_ref
    assert it_ours == it_ref
    np.testing.assert_allclose(_dist(ours, n, k), _dist(refd, n, k), rtol=1e-10, atol=0)


def test_main_baa_resumes_from_its_saved_distribution(tmp_path, O):
    # stop after a fixed number of iterations (a = 0.05), then resume from the
    # saved file with a tighter a: the same as one uninterrupted run
    n, k = 10, 5
    d = _workdir(tmp_path, "ours", OUR_GEN, (n + 1) // 2)
    _run(OUR_MAIN, d, n, k, 0, 0.05, 1000)
    first = _dist(d, n, k)
    _, line = _summary(_run(OUR_MAIN, d, n, k, 1, 1e-3, 1000))
    reps = O.canonicals(n)
    r1 = O.run_ba(n, k, np.full(len(reps), 1.0 / (1 << n)), reps, 0.05, 100000)
    np.testing.assert_allclose(first, r1["p"], rtol=1e-10, atol=0)
    r2 = O.run_ba(n, k, r1["p"], reps, 1e-3, 100000)
    np.testing.assert_allclose(_dist(d, n, k), r2["p"], rtol=1e-10, atol=0)
    assert line == f"Computed C_{{{n},{k}}} = {r2['rate_bits']:.6f} bits (max deviation {r2['mx_final']:.6f})"


def test_main_baa_device_tables_and_errors(tmp_path, O):
    n, k = 9, 4
    d = tmp_path / "dev"
    (d / "distributions").mkdir(parents=True)
    env = dict(os.environ, BDC_TABLES="device")
    r = subprocess.run([OUR_MAIN, str(n), str(k), "0", "1e-3", "1000"], cwd=d, env=env,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    reps = O.canonicals(n)
    ref = O.run_ba(n, k, np.full(len(reps), 1.0 / (1 << n)), reps, 1e-3, 100000)
    np.testing.assert_allclose(_dist(d, n, k), ref["p"], rtol=1e-10, atol=0)
    # a distribution file of the wrong length is an error, not a silent run
    (d / "distributions" / f"dist_{n}_{k}.txt").write_text("0.5\n0.5\n")
    r = subprocess.run([OUR_MAIN, str(n), str(k), "1"], cwd=d, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 2
    # missing tables: error exit, like the reference's try_to_open_file
    shutil.rmtree(d / "distributions")
    (d / "distributions").mkdir()
    r = subprocess.run([OUR_MAIN, str(n), str(k)], cwd=d, capture_output=True, text=True, timeout=300)
    assert r.returncode != 0


def test_main_baa_certified_solver_mode(tmp_path, O):
    # BDC_SOLVE=<gap>: the certified solver instead of the plain loop; the
    # saved distribution carries the printed lower end of the bracket
    n, k = 12, 6
    d = tmp_path / "solve"
    (d / "distributions").mkdir(parents=True)
    env = dict(os.environ, BDC_TABLES="device", BDC_SOLVE="1e-9")
    r = subprocess.run([OUR_MAIN, str(n), str(k)], cwd=d, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    m = re.search(r"^Certified C_\{12,6\} in \[(\S+), (\S+)\] bits", r.stdout, re.M)
    assert m, r.stdout
    lo, hi = float(m.group(1)), float(m.group(2))
    assert 0.0 <= hi - lo < 1e-9
    p = _dist(d, n, k)
    reps = O.canonicals(n)
    lnq = O.log_q(n, k, p, reps)
    assert abs(O.rate(n, k, lnq, p, reps) / np.log(2.0) - lo) < 1e-11
