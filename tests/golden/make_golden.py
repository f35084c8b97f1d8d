"""Generates the golden fixtures of tests/golden from the reference's own programs.

Test infrastructure: runs the reference programs compiled unchanged by
oracle/Makefile (`make -C oracle ref`) into oracle/_ref/.

  python tests/golden/make_golden.py caches [--max-n 10]
      runs the reference cache generator (backend/generate_bit_transition_cache.cpp)
      for all n' <= max_n, k' < n' in a scratch directory and writes
      ref_cache_sha256.json (sha256 of every cache_n_k file) and copies the
      small files cache_{n}_{k} with n <= 6 verbatim into ref_caches/.

  python tests/golden/make_golden.py ba --out DIR
      (needs a GPU) runs oracle/_ref/ref_harness, i.e. the reference's
      backend/BAA.cu host API, on the configurations in CONFIGS and packs the
      full-precision vectors into DIR/ref_ba_<name>.npz.  Vectors longer than
      SAMPLE_CAP are stored as a seeded sample of indices plus full-vector
      checksums (sum, sum of squares, max) so that the fixtures stay small.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_BIN = os.path.join(REPO, "oracle", "_ref")
sys.path.insert(0, os.path.join(REPO, "bdc-upper-bounds-gpu_b200"))

SAMPLE_CAP = 20000

# name, n, k, iterations, start
CONFIGS = [
    ("n3k2_uniform", 3, 2, 6, ("uniform",)),
    ("n8k8_uniform", 8, 8, 3, ("uniform",)),
    ("n9k1_uniform", 9, 1, 4, ("uniform",)),
    ("n10k4_dirichlet05_s3", 10, 4, 6, ("dirichlet", 0.5, 3)),
    ("n10k5_zeros", 10, 5, 4, ("zeros", 1.0, 7)),
    ("n12k6_uniform", 12, 6, 12, ("uniform",)),
    ("n13k5_uniform", 13, 5, 6, ("uniform",)),
    ("n13k7_dirichlet1_s1", 13, 7, 6, ("dirichlet", 1.0, 1)),
    ("n16k8_dirichlet1_s0", 16, 8, 4, ("dirichlet", 1.0, 0)),
    ("n20k10_dirichlet1_s0", 20, 10, 3, ("dirichlet", 1.0, 0)),
    ("n24k12_uniform", 24, 12, 2, ("uniform",)),
]


def sha256(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 20), b""):
            h.update(chunk)
    return h.hexdigest()


def cmd_caches(max_n: int) -> None:
    gen = os.path.join(REF_BIN, "generate_bit_transition_cache")
    with tempfile.TemporaryDirectory() as td:
        os.makedirs(os.path.join(td, "transition_counts"))
        subprocess.run([gen, str(max_n)], cwd=td, check=True)
        out = {}
        small = os.path.join(HERE, "ref_caches")
        os.makedirs(small, exist_ok=True)
        for n in range(1, max_n + 1):
            for k in range(0, n):
                p = os.path.join(td, "transition_counts", f"cache_{n}_{k}")
                out[f"cache_{n}_{k}"] = sha256(p)
                if n <= 6:
                    shutil.copy(p, os.path.join(small, f"cache_{n}_{k}"))
    with open(os.path.join(HERE, "ref_cache_sha256.json"), "w") as f:
        json.dump({"generator": "backend/generate_bit_transition_cache.cpp (reference, unchanged)",
                   "max_n": max_n, "sha256": out}, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} hashes")


def start_vector(n: int, spec) -> np.ndarray | None:
    from bdc_b200.dist import dirichlet_start
    if spec[0] == "uniform":
        return None
    if spec[0] == "dirichlet":
        return dirichlet_start(n, spec[1], spec[2])
    if spec[0] == "zeros":
        # Dirichlet start with every 5th representative set to 0 and no
        # renormalisation: exercises the reference's ln 0 = 0 rule and its
        # lack of input normalisation (backend/BAA.cu:573-580, main_BAA.cu:59-61)
        p = dirichlet_start(n, spec[1], spec[2])
        p[::5] = 0.0
        return p
    raise ValueError(spec)


def pack(vec: np.ndarray, rng: np.random.Generator) -> dict:
    if len(vec) <= SAMPLE_CAP:
        return {"full": vec}
    idx = np.sort(rng.choice(len(vec), SAMPLE_CAP, replace=False))
    return {"idx": idx.astype(np.int64), "val": vec[idx],
            "sum": np.sum(vec), "sumsq": np.sum(vec * vec), "max": np.max(vec)}


def cmd_ba(out_dir: str, names: list[str] | None) -> None:
    harness = os.path.join(REF_BIN, "ref_harness")
    gen = os.path.join(REF_BIN, "generate_bit_transition_cache")
    os.makedirs(out_dir, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        os.makedirs(os.path.join(td, "transition_counts"))
        max_half = max((c[1] + 1) // 2 for c in CONFIGS if not names or c[0] in names)
        subprocess.run([gen, str(max_half)], cwd=td, check=True)
        for name, n, k, iters, spec in CONFIGS:
            if names and name not in names:
                continue
            run = os.path.join(td, name)
            os.makedirs(run)
            p0 = start_vector(n, spec)
            init = "uniform"
            if p0 is not None:
                init = os.path.join(run, "p_init.bin")
                p0.astype("<f8").tofile(init)
            with open(os.path.join(out_dir, f"ref_ba_{name}.log"), "w") as log:
                subprocess.run([harness, str(n), str(k), str(iters), init, run], cwd=td,
                               stdout=log, stderr=subprocess.STDOUT, check=True)
            meta = open(os.path.join(run, "meta.txt")).read().split("\n")
            mx = [float(l.split()[3]) for l in meta if l.startswith("iter ")]
            tms = [float(l.split()[2]) for l in meta if l.startswith("time_iter_s ")]
            rate = [float(l.split()[1]) for l in meta if l.startswith("rate_nats ")][0]
            rng = np.random.default_rng(12345)
            arrays = {"n": n, "k": k, "iters": iters, "mx": np.array(mx), "rate_nats": rate,
                      "time_iter_s": np.array(tms), "start": str(spec)}
            def rd(f):
                return np.fromfile(os.path.join(run, f), dtype="<f8")
            vecs = {"p_0": rd("p_0.bin"), "kl_final": rd("kl_final.bin"), "lnq_final": rd("lnq_final.bin")}
            for t in range(iters):
                vecs[f"lnq_{t}"] = rd(f"lnq_{t}.bin")
                vecs[f"logw_{t}"] = rd(f"logw_{t}.bin")
                vecs[f"p_{t + 1}"] = rd(f"p_{t + 1}.bin")
            for key, v in vecs.items():
                for sub, val in pack(v, rng).items():
                    arrays[f"{key}.{sub}"] = val
            np.savez_compressed(os.path.join(out_dir, f"ref_ba_{name}.npz"), **arrays)
            print(name, "iters", iters, "rate_nats", rate, "mx", mx[-1])


def main() -> None:
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    a = sub.add_parser("caches")
    a.add_argument("--max-n", type=int, default=10)
    b = sub.add_parser("ba")
    b.add_argument("--out", default=HERE)
    b.add_argument("--only", nargs="*")
    args = ap.parse_args()
    if args.cmd == "caches":
        cmd_caches(args.max_n)
    else:
        cmd_ba(args.out, args.only)


if __name__ == "__main__":
    main()
