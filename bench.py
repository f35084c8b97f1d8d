"""Benchmark of the Blahut-Arimoto engine on BDC_{24,12}.

One step = one BA iteration over all 4,196,352 canonical representatives of
{0,1}^24 with output length 12 (the q pass, the D pass and the normalised
update with its stopping statistic), starting from the uniform distribution.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  Under torchrun (N > 1) every rank runs an
independent replica (BA on one (n,k) does not shard across GPUs in this
build) and the reported value is the total iterations/s of all replicas.

--impl reference times the reference's own CPU implementation of the path on
the host cores: the reference has no CPU BA, so this is the CPU oracle port
(oracle/bdc_oracle.c, OpenMP over all cores) on a bounded sample of
representatives, extrapolated to all representatives per iteration.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "bdc-upper-bounds-gpu_b200"))

METRIC = "BA iters/s & time-to-bound (1e-9 bits) at n=24,k=12: accelerated vs plain BA"
UNIT = "BA iterations/s"
FALLBACK_PEAKS = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def load_peaks() -> tuple[dict, str]:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return json.load(open(p)), "measured"
    return dict(FALLBACK_PEAKS), "fallback"


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampled every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def profile_traffic(kernel: str, n: int, k: int):
    """DRAM bytes per launch of `kernel` at (n, k) from the committed ncu
    summaries (profiles/*.md lines "traffic <kernel> <n> <k> <bytes>"), or None."""
    d = os.path.join(REPO, "profiles")
    if not os.path.isdir(d):
        return None
    for f in sorted(os.listdir(d)):
        if not f.endswith((".md", ".txt")):
            continue
        for line in open(os.path.join(d, f)):
            w = line.strip().strip("`").split()
            if len(w) == 5 and w[0] == "traffic" and w[1] == kernel and w[2] == str(n) and w[3] == str(k):
                return float(w[4])
    return None


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def reference_cuda_leg(n: int, k: int, iters: int = 2) -> dict:
    """The reference's own CUDA BA on this GPU: backend/BAA.cu compiled
    unchanged (oracle/_ref/ref_harness, built by oracle/Makefile from the
    reference sources), driven through its host API from the uniform start.
    The harness times baa_iteration + compute_max_deviation (the body of the
    reference loop, main_BAA.cu:80-99) with CUDA events; the cache files it
    loads (transition_counts/cache_{n',k'}, n' <= ceil(n/2)) are written by
    this repository's generator, byte-identical to the reference's."""
    import shutil
    harness = os.path.join(REPO, "oracle", "_ref", "ref_harness")
    gen = os.path.join(REPO, "bdc-upper-bounds-gpu_b200", "generate_bit_transition_cache")
    if not (os.path.exists(harness) and os.path.exists(gen)):
        return {"unavailable": "oracle/_ref/ref_harness not built (make -C oracle ref)"}
    d = tempfile.mkdtemp(prefix="bdc_refcuda_")
    try:
        os.makedirs(os.path.join(d, "transition_counts"))
        subprocess.run([gen, str((n + 1) // 2)], cwd=d, check=True, stdout=subprocess.DEVNULL, timeout=300)
        out = os.path.join(d, "out")
        os.makedirs(out)
        t0 = time.perf_counter()
        r = subprocess.run([harness, str(n), str(k), str(iters), "uniform", out], cwd=d, capture_output=True,
                           text=True, timeout=600)
        wall = time.perf_counter() - t0
        if r.returncode != 0:
            return {"unavailable": f"ref_harness exited {r.returncode}: {r.stderr.strip()[-200:]}"}
        times = [float(line.split()[2]) for line in open(os.path.join(out, "meta.txt"))
                 if line.startswith("time_iter_s")]
        sec = float(np.median(times))
        return {"seconds_per_iteration": sec, "iterations_per_s": 1.0 / sec, "iterations_timed": len(times),
                "per_iteration_s": times, "harness_wall_s": wall,
                "what": "reference backend/BAA.cu compiled unchanged for sm_100a (oracle/_ref/ref_harness), "
                        "CUDA events around baa_iteration + compute_max_deviation, uniform start, same GPU"}
    except (subprocess.SubprocessError, OSError, ValueError) as e:
        return {"unavailable": f"{type(e).__name__}: {e}"[:200]}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def cpu_full_iteration(n: int, k: int) -> dict:
    """One whole BA iteration of the CPU oracle port (the reference's
    per-representative algorithm: per-x DP, distinct subsequences, split
    identity, orbit factors) over every representative, all host threads,
    from the uniform start; measured, not extrapolated."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    reps = O.canonicals(n)
    p = np.full(len(reps), 1.0 / (1 << n))
    O.log_q(n, k, p[:8], reps[:8])  # builds the cached half tables (not timed)
    t0 = time.perf_counter()
    O.ba_iteration(n, k, p, reps)
    sec = time.perf_counter() - t0
    return {"n": n, "k": k, "representatives": int(len(reps)), "seconds_per_iteration": sec,
            "iterations_per_s": 1.0 / sec, "cores": O.threads(), "kind": "port", "cpu_model": cpu_model()}


# --------------------------------------------------------------- CPU legs
def cpu_ba_iteration_rate(n: int, k: int, sample: int, threads: int | None = None) -> dict:
    """The CPU oracle's q pass + D pass on `sample` evenly spaced
    representatives, extrapolated to all of them, plus the O(R) update.
    Returns iterations/s, the threads used and a description."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle as O
    if threads:
        O.set_threads(threads)
    reps = O.canonicals(n)
    R = len(reps)
    idx = np.linspace(0, R - 1, min(sample, R)).astype(np.int64)
    sub = reps[idx]
    p = np.full(len(sub), 1.0 / (1 << n))
    O.log_q(n, k, p[:8], sub[:8])  # builds the cached half tables (not timed)
    t0 = time.perf_counter()
    lnq = O.log_q(n, k, p, sub)
    t1 = time.perf_counter()
    O.log_w(n, k, p, lnq, sub)
    t2 = time.perf_counter()
    pf = np.full(R, 1.0 / (1 << n))
    lw = np.log(pf) + 1.0
    t3 = time.perf_counter()
    O.normalise(n, lw, reps)
    t4 = time.perf_counter()
    per_iter = (t2 - t0) * (R / len(sub)) + (t4 - t3)
    return {"value": 1.0 / per_iter, "unit": UNIT, "cores": O.threads(),
            "sample": f"q pass + D pass on {len(sub)} of {R} representatives (evenly spaced), "
                      f"scaled by {R / len(sub):.1f}, plus the full O(R) normalisation; "
                      f"{t2 - t0:.2f} s of sampled CPU work",
            "seconds_per_iteration": per_iter, "representatives": int(R), "sampled": int(len(sub)),
            "fraction": len(sub) / R}


def workload_config(n: int, k: int, R: int) -> dict:
    """The workload both arms report (same keys and values in both lines)."""
    return {"workload": f"BA iteration on BDC_{{{n},{k}}}", "n": n, "k": k, "representatives": R,
            "start": "uniform", "parallelism": "replicas x1",
            "l2": "working set per iteration > L2 (p, D, logW, h vectors of 33.6 MB each + 32 MB tables)"}


def reference_arm(args) -> None:
    """The reference's algorithm on the host cores.  The reference's BA runs
    only on a GPU (backend/BAA.cu); its CPU restatement (oracle/bdc_oracle.c:
    per-x DP, distinct subsequences, split identity, orbit factors, OpenMP
    over all host threads) stands in.  Each step is a bounded sample of one
    iteration: the q and D passes over `cpu_sample` evenly spaced
    representatives plus the full O(R) normalisation.  ms_per_step is the
    measured time of that sampled step; value is the whole-iteration rate it
    implies (the sampled passes scaled to every representative)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    steps, walls = [], []
    meta = None
    for _ in range(max(1, args.warmup)):
        cpu_ba_iteration_rate(args.n, args.k, args.cpu_sample)
    for _ in range(args.steps):
        t0 = time.perf_counter()
        meta = cpu_ba_iteration_rate(args.n, args.k, args.cpu_sample)
        walls.append(time.perf_counter() - t0)
        steps.append(1.0 / meta["value"])
    sec = float(np.mean(steps))
    v = 1.0 / sec
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(walls)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (uniform start; the reference publishes no throughput)",
        "config": workload_config(args.n, args.k, meta["representatives"]),
        "engine": "cpu port of the reference's per-representative algorithm (oracle/bdc_oracle.c, OpenMP)",
        "sampled_step": {"representatives_sampled": meta["sampled"], "fraction": meta["fraction"],
                         "ms_per_full_iteration_extrapolated": sec * 1e3},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": meta["cores"], "kind": "port",
                         "sample": meta["sample"], "cpu_model": cpu_model()},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU BA implementation (its BA is CUDA); this is the CPU restatement of its "
                "BA iteration on all host threads; each step is a bounded sample, value is the full-iteration rate",
    }
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------- GPU leg
def ours_arm(args) -> None:
    import torch

    import bdc_b200

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    stream = torch.cuda.current_stream()
    E = bdc_b200.Engine(args.n, args.k, engine=args.engine, device=local)
    E.set_stream(stream.cuda_stream)
    E.set_uniform()
    R = E.R
    pairs, S = E.work()

    # warm-up, then K iterations timed with events on the stream the engine uses
    # warm-up (at least 16 iterations, so that the captured iteration graph
    # exists before timing)
    E.iterate(max(args.warmup, 16), float("-inf"))
    prof = E.profile(2)
    launches_per_iter = prof["launches"]
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        st = E.iterate(args.steps, float("-inf"))
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms = max_over_ranks(e0.elapsed_time(e1))
    clocks = clk.summary()
    assert st["iters"] == args.steps
    value = world * args.steps / (ms / 1e3)

    # end to end through the reference-shaped call: pinned host p in, p' out
    p_in = torch.empty(R, dtype=torch.float64, pin_memory=True)
    p_out = torch.empty(R, dtype=torch.float64, pin_memory=True)
    p_in.fill_(1.0 / (1 << args.n))
    for _ in range(max(1, min(args.warmup, 3))):
        E.baa_iteration_ptr(p_in.data_ptr(), p_out.data_ptr())
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_steps = max(1, min(args.steps, 50))
    f0.record(stream)
    for _ in range(e2e_steps):
        E.baa_iteration_ptr(p_in.data_ptr(), p_out.data_ptr())
        p_in, p_out = p_out, p_in
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1))
    e2e = {"value": world * e2e_steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": R * 8, "d2h_bytes_per_step": R * 8,
           "call": "bdc_baa_iteration (host p in, host p' out)"}
    # the copies alone (pinned, same sizes): the end-to-end bound is one H2D,
    # one iteration and one D2H in sequence (each call depends on the last)
    d_buf = torch.empty(R, dtype=torch.float64, device="cuda")
    h2d, d2h = [], []
    for _ in range(5):
        c0, c1, c2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        c0.record(stream)
        d_buf.copy_(p_in, non_blocking=True)
        c1.record(stream)
        p_out.copy_(d_buf, non_blocking=True)
        c2.record(stream)
        torch.cuda.synchronize()
        h2d.append(c0.elapsed_time(c1))
        d2h.append(c1.elapsed_time(c2))
    h2d_ms, d2h_ms = float(np.median(h2d)), float(np.median(d2h))
    bound_ms = h2d_ms + ms / args.steps + d2h_ms
    e2e.update({"pcie_h2d_gbs": R * 8 / (h2d_ms / 1e3) / 1e9, "pcie_d2h_gbs": R * 8 / (d2h_ms / 1e3) / 1e9,
                "bound": world * 1e3 / bound_ms, "frac": (world * e2e_steps / (e2e_ms / 1e3)) / (world * 1e3 / bound_ms),
                "bound_model": "median pinned H2D + device iteration + D2H, measured in this run"})
    del d_buf

    # roofline of the dominant kernel, with measured pipe peaks
    peaks, peak_src = load_peaks()
    imad = bdc_b200.peak_probe("imad", local)
    dfma = bdc_b200.peak_probe("dfma", local)
    if E.engine == "count":
        achieved = prof["work_main"] / (prof["ms_main"] / 1e3)
        roofline = {"bound": "int32 multiply-add pipe (no tensor cores: exact integer counts)",
                    "kernel": "k_dpass (D pass; the q pass k_qpass is the same count loop)",
                    "achieved": achieved / 1e12, "peak": imad / 1e12, "unit": "Tops/s",
                    "frac": achieved / imad, "traffic": None,
                    "work_per_launch": f"{pairs} nonzero (x,y) pairs x {S} split terms = "
                                       f"{prof['work_main']:.4e} multiply-adds",
                    "peak_source": "bdc_peak_probe int32 IMAD chain, measured in this run"}
    elif prof["main_kind"] == 2:
        # the G stage on the int8 tensor cores (k_oz_ba, the exact split of its
        # FP64 operands): its tensor work is small, its bound is the update's
        # device-memory traffic; ms_main is its CUDA-event time per iteration
        achieved = prof["bytes_main"] / (prof["ms_main"] / 1e3) / 1e9
        roofline = {"bound": "hbm",
                    "kernel": "k_oz_ba (G = [A_L | N_R] [M_L ; B_R^T] as eight exact int8 products on tcgen05.mma "
                              "kind::i8, TMEM accumulators, BA update in the epilogue)",
                    "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                    "frac": achieved / peaks.get("hbm_gbs"), "traffic": profile_traffic("k_oz_ba", args.n, args.k),
                    "work_per_launch": f"40 bytes per representative (read h, ln p, p; write ln p, p) x R = "
                                       f"{prof['bytes_main']:.4e} bytes",
                    "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_src})"}
    else:
        # the G stage: one k_mma_ba launch (FP64 mma.sync tiles, the BA update
        # fused in the epilogue); ms_main is its CUDA-event time per iteration
        achieved = prof["work_main"] / (prof["ms_main"] / 1e3)
        dmma = bdc_b200.peak_probe("dmma", local)
        roofline = {"bound": "tensor",
                    "kernel": "k_mma_ba (G = [A_L | N_R] [M_L ; B_R^T] on FP64 mma.sync, BA update in the epilogue)",
                    "achieved": achieved / 1e12, "peak": 2 * dmma / 1e12, "unit": "TFLOP/s",
                    "frac": achieved / (2 * dmma), "traffic": profile_traffic("k_mma_ba", args.n, args.k),
                    "work_per_launch": f"2*R*K = {prof['work_main']:.4e} flops: one K-long dot product per "
                                       f"representative (R = {R}, K = sum of the split-term widths); the "
                                       f"launch executes the tiles that hold representatives, 1.07x that",
                    "peak_source": "bdc_peak_probe FP64 mma.sync m8n8k4 chains on all SMs, measured in this "
                                   "run (2 flops per multiply-add); MEASURED_PEAKS.json holds no FP64 figure"}
    upd_bytes = R * 72
    roofline_update = None if E.engine != "count" else {"bound": "hbm", "achieved": upd_bytes / (prof["ms_update"] / 1e3) / 1e9,
                       "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                       "frac": upd_bytes / (prof["ms_update"] / 1e3) / 1e9 / peaks.get("hbm_gbs"),
                       "traffic": None, "peak_source": f"MEASURED_PEAKS.json hbm_gbs ({peak_src})",
                       "work_per_launch": "72 bytes per representative over the three update kernels"}

    ttb = None
    if world == 1 and not args.no_ttb and E.engine == "factored":
        ttb = time_to_bound(args, E)

    cpu = None
    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_ba_iteration_rate(args.n, args.k, max(args.cpu_sample, 50000))
        cpu = {k2: cpu[k2] for k2 in ("value", "unit", "cores", "sample")} | {
            "kind": "port", "cpu_model": cpu_model(), "extrapolated": True}
        # a whole iteration, measured, at the largest size the CPU finishes in
        # seconds, next to this engine's iteration at the same size
        full = cpu_full_iteration(20, 10)
        with bdc_b200.Engine(20, 10, engine="auto", device=local) as E20:
            E20.set_stream(stream.cuda_stream)
            E20.set_uniform()
            E20.iterate(16, float("-inf"))
            torch.cuda.synchronize()
            g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g0.record(stream)
            E20.iterate(200, float("-inf"))
            g1.record(stream)
            torch.cuda.synchronize()
            full["gpu_iterations_per_s"] = 200 / (g0.elapsed_time(g1) / 1e3)
            full["gpu_engine"] = E20.engine
        cpu["full_iteration_20_10"] = full
        cpu["cache_generator"] = generator_leg(11)
    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        import copy
        a5 = copy.copy(args)
        a5.n, a5.k, a5.fd_seeds, a5.fd_coords = 26, 13, 16, 64
        configs = {"config4_batched_time_to_bound": batch_time_to_bound(2, 1e-9, local),
                   "config5_adjoint_26_13": adjoint_check(a5)}
    if rank == 0 and world == 1 and not args.no_ref_cuda:
        ref_cuda = reference_cuda_leg(args.n, args.k, 2)
        if "seconds_per_iteration" in ref_cuda:
            ref_cuda["speedup_of_value"] = value * ref_cuda["seconds_per_iteration"]
            ref_cuda["speedup_of_e2e"] = e2e["value"] * ref_cuda["seconds_per_iteration"]

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (uniform start; the reference publishes no throughput)",
        "config": workload_config(args.n, args.k, R) | {"parallelism": f"replicas x{world}"},
        "engine": E.engine,
        "g_product": {0: None, 1: "FP64 mma.sync", 2: "int8 tcgen05 (exact split)"}[prof["main_kind"]],
        "gpu_launches": launches_per_iter * args.steps,
        "profile_ms": {k2: prof[k2] for k2 in ("ms_q", "ms_fold", "ms_d", "ms_update", "ms_iter", "ms_main")},
        "roofline": roofline, "roofline_update": roofline_update,
        "peaks_measured": {"int32_madd_tops": imad / 1e12, "fp64_fma_tflops": 2 * dfma / 1e12,
                           "hbm_gbs": peaks.get("hbm_gbs"), "hbm_source": peak_src},
        "e2e": e2e, "cpu_baseline": cpu, "reference_gpu": ref_cuda, "clocks": clocks, "time_to_bound": ttb,
        "configs": configs,
        "bound_bits": st["upper_bound"], "rate_bits": st["rate"],
    }
    E.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def time_to_bound(args, E=None) -> dict:
    """Time-to-bound at (n, k) from the uniform start, tolerance 1e-9 bits.

    The certified solver (bdc_solve) returns a bracket rate <= C <= bound,
    both evaluated at its final point; its time is the CUDA-event time of the
    call (the median of three solves).  The accelerated loop (bdc_accelerate:
    Nesterov-accelerated exponentiated gradient driven by the adjoint) runs
    from the uniform start in one call until its own bracket is below 1e-9
    bits, which proves its bound within 1e-9 bits of C.  Plain BA runs from
    the uniform start in chunks for at most `budget` seconds of device time;
    it has reached the bound when its best upper bound is within 1e-9 bits
    of C, i.e. best_ub - certified rate < 1e-9 (C >= that rate)."""
    import torch

    import bdc_b200

    tol = 1e-9
    own = E is None
    if own:
        E = bdc_b200.Engine(args.n, args.k, engine="factored")
    stream = torch.cuda.current_stream()
    E.set_stream(stream.cuda_stream)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        r = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return r, e0.elapsed_time(e1) / 1e3

    # warm-up: the iteration graph, the accelerated step graph and one solve
    E.set_uniform()
    E.accelerate(48, 0.0)
    E.set_uniform()
    E.iterate(16, float("-inf"))
    E.set_uniform()
    E.solve(1e-6, 20000)
    solves = []
    for _ in range(3):
        E.set_uniform()
        st, sec = timed(lambda: E.solve(tol, 200000))
        solves.append((sec, st))
    solves.sort(key=lambda v: v[0])
    sec, st = solves[1]
    lo, hi = st["best_rate"], st["best_upper_bound"]
    out = {"tolerance_bits": tol, "C_bracket_bits": [lo, hi],
           "certified": {"seconds": sec, "seconds_of_three": [v[0] for v in solves],
                         "full_evaluations": st["iters"], "gap_bits": hi - lo, "reached": bool(hi - lo < tol)}}
    # accelerated: one call to its own certified bracket
    E.set_uniform()
    max_evals = int(args.ttb_budget / 2.5e-4)
    sa, seca = timed(lambda: E.accelerate(max_evals, tol))
    out["accelerated"] = {"method": "Nesterov-accelerated exponentiated gradient, adaptive restart (bdc_accelerate)",
                          "seconds": seca, "evaluations": sa["iters"],
                          "bracket_bits": sa["best_upper_bound"] - sa["best_rate"],
                          "bound_minus_C_bits_at_most": sa["best_upper_bound"] - lo,
                          "reached": bool(sa["converged"])}
    # plain BA for the budget
    E.set_uniform()
    evals, total = 0, 0.0
    chunk = 64
    reached = False
    best = None
    trace = []  # (seconds, best bound - C) after each chunk
    while total < args.ttb_budget:
        sp, secp = timed(lambda: E.iterate(chunk, float("-inf")))
        total += secp
        evals += sp["iters"]
        best = sp["best_upper_bound"]
        trace.append((total, best - lo))
        if best - lo < tol:
            reached = True
            break
        chunk = min(chunk * 2, 4096)
    leg = {"budget_s": args.ttb_budget, "seconds": total, "evaluations": evals, "reached": reached,
           "bound_minus_C_bits_at_most": best - lo}
    if not reached:
        # extrapolated, and labelled so: the gap's decay over the second half
        # of the run, taken as exponential in time, continued to 1e-9 bits
        half = [(t, g) for t, g in trace if t >= total / 2 and g > 0]
        if len(half) >= 2 and half[-1][1] < half[0][1]:
            rate = (math.log(half[0][1]) - math.log(half[-1][1])) / (half[-1][0] - half[0][0])
            leg["extrapolated_seconds_to_1e-9"] = total + math.log(half[-1][1] / tol) / rate
    out["plain"] = leg
    for name in ("certified", "accelerated"):
        if not out[name]["reached"]:
            continue
        t = out[name]["seconds"]
        if reached:
            out[name]["speedup_vs_plain"] = total / t
        else:
            out[name]["speedup_vs_plain_at_least"] = total / t
            if "extrapolated_seconds_to_1e-9" in leg:
                out[name]["speedup_vs_plain_extrapolated"] = leg["extrapolated_seconds_to_1e-9"] / t
    if own:
        E.close()
    return out


BATCH_MIX = [(16, 8), (18, 6), (20, 10), (22, 11), (24, 8), (24, 12)]


def batched(args) -> dict | None:
    """The batched form: the six (n,k) instances of BATCH_MIX x 8 seeds of a
    Dirichlet(0.5) start (48 BA instances), iterated together from one
    captured CUDA graph, against the same engines iterated one after the
    other.  Both legs run the same number of BA iterations per instance with
    no stopping threshold; the figure is instance-iterations per second.
    Under torchrun the instances are spread over the ranks (replicas, no
    data-path collective) and the time is the max over ranks."""
    import torch

    import bdc_b200
    from bdc_b200 import dist as bdist
    from bdc_b200 import replicas

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    tdist = None
    if world > 1:
        import datetime

        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
    seeds = range(8)
    mix = [(n, k, s) for n, k in BATCH_MIX for s in seeds]
    mine = replicas.partition([(n, k) for n, k, _ in mix], world)[rank]
    engines = []
    for i in mine:
        n, k, s = mix[i]
        E = bdc_b200.Engine(n, k, engine="factored", device=local)
        E.set_p(bdist.dirichlet_start(n, 0.5, s))
        engines.append(E)
    stream = torch.cuda.current_stream()
    iters = max(args.steps, 8)
    B = bdc_b200.Batch(engines)
    B.set_stream(stream.cuda_stream)
    B.iterate(16, float("-inf"))  # warm-up: captures the batch graph
    for E in engines:
        E.set_stream(stream.cuda_stream)
        E.iterate(16, float("-inf"))  # warm-up: each engine's own graph
    torch.cuda.synchronize()

    def max_over_ranks(v: float) -> float:
        if tdist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
        return float(t.item())

    def timed(fn) -> float:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if tdist is not None:
            tdist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1) / 1e3)

    t_batch = timed(lambda: B.iterate(iters, float("-inf")))
    t_seq = timed(lambda: [E.iterate(iters, float("-inf")) for E in engines])
    per_nk = {}
    if world == 1:
        for i, (n, k) in enumerate(BATCH_MIX):
            E = engines[i * len(seeds)]
            per_nk[f"{n}_{k}"] = iters / timed(lambda: E.iterate(iters, float("-inf")))
    total = len(mix) * iters
    ttb8 = batch_time_to_bound(len(seeds), 1e-9, local) if world == 1 else None
    out = {"instances": len(mix), "n_gpus": world, "iters_per_instance": iters, "time_to_bound": ttb8,
           "batched_instance_iters_per_s": total / t_batch,
           "sequential_instance_iters_per_s": total / t_seq,
           "batch_speedup": t_seq / t_batch,
           "single_engine_iters_per_s": per_nk}
    B.close()
    for E in engines:
        E.close()
    if tdist is not None:
        tdist.destroy_process_group()
    return out if rank == 0 else None


def batch_time_to_bound(seeds: int, gap: float = 1e-9, device: int = 0) -> dict:
    """Per-instance time-to-bound of the batched accelerated loop: the
    instances of BATCH_MIX x `seeds` Dirichlet(0.5) starts iterated together
    from one captured graph (bdc_batch_accelerate), each stopping on its own
    certified bracket < gap bits.  An instance's time is the device time from
    the batch's start until its bracket fell below gap (resolution: one graph
    replay of 8 steps of every live instance)."""
    import torch

    import bdc_b200
    from bdc_b200 import dist as bdist

    engines, names = [], []
    for n, k in BATCH_MIX:
        for sd in range(seeds):
            E = bdc_b200.Engine(n, k, engine="factored", device=device)
            E.set_p(bdist.dirichlet_start(n, 0.5, sd))
            engines.append(E)
            names.append((n, k, sd))
    B = bdc_b200.Batch(engines)
    B.set_stream(torch.cuda.current_stream().cuda_stream)
    B.accelerate(16, 0.0)  # warm-up: captures the batch's step graph
    for E, (n, k, sd) in zip(engines, names):
        E.set_p(bdist.dirichlet_start(n, 0.5, sd))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    stats, secs = B.accelerate(400000, gap)
    wall = time.perf_counter() - t0
    inst = []
    for (n, k, sd), st, sec in zip(names, stats, secs):
        inst.append({"n": n, "k": k, "seed": sd, "seconds_to_bracket": sec, "evaluations": st["iters"],
                     "bracket_bits": st["best_upper_bound"] - st["best_rate"],
                     "upper_bound_bits": st["best_upper_bound"], "reached": bool(st["converged"])})
    B.close()
    for E in engines:
        E.close()
    return {"instances": len(inst), "gap_bits": gap, "start": "Dirichlet(0.5), seeds 0.." + str(seeds - 1),
            "all_reached": all(i["reached"] for i in inst), "batch_seconds": max(i["seconds_to_bracket"] for i in inst),
            "wall_seconds": wall, "per_instance": inst}


def adjoint_check(args) -> dict:
    """The adjoint at (n, k) (default 26/13): for each of `fd_seeds` Dirichlet(1)
    starts, dI/dp from bdc_mi_backward against central differences of
    bdc_mi_forward with h = 1e-7 on `fd_coords` seeded coordinates; the
    iterate moves device to device (bdc_set_p_device), one coordinate at a
    time.  Reports the largest error relative to max(1, |dI/dp|) and the time
    of one forward and one backward evaluation."""
    import torch

    import bdc_b200
    from bdc_b200 import dist as bdist

    h = 1e-7
    E = bdc_b200.Engine(args.n, args.k, engine="factored")
    stream = torch.cuda.current_stream()
    E.set_stream(stream.cuda_stream)
    out = {"n": args.n, "k": args.k, "h": h, "coords_per_seed": args.fd_coords, "seeds": args.fd_seeds,
           "max_rel_err": 0.0, "per_seed": []}
    t_fwd, t_bwd = [], []
    for seed in range(args.fd_seeds):
        p = torch.from_numpy(bdist.dirichlet_start(args.n, 1.0, seed)).cuda()
        E.set_p_device(p.data_ptr())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = E.mi_backward()
        t_bwd.append(time.perf_counter() - t0)
        rng = np.random.default_rng(seed)
        idx = rng.choice(E.R, args.fd_coords, replace=False)
        worst = 0.0
        for i in idx:
            i = int(i)
            v = float(p[i])
            p[i] = v + h
            E.set_p_device(p.data_ptr())
            t0 = time.perf_counter()
            ip = E.mi_forward(None)
            t_fwd.append(time.perf_counter() - t0)
            p[i] = v - h
            E.set_p_device(p.data_ptr())
            im = E.mi_forward(None)
            p[i] = v
            fd = (ip - im) / (2 * h)
            worst = max(worst, abs(fd - g[i]) / max(1.0, abs(g[i])))
        out["per_seed"].append(worst)
        out["max_rel_err"] = max(out["max_rel_err"], worst)
    out["forward_ms_median"] = 1e3 * float(np.median(t_fwd))
    out["backward_ms_median"] = 1e3 * float(np.median(t_bwd))
    E.close()
    return out


def precision_check(args) -> dict:
    """The precision form: the count path with FP64 sums against the same path
    with compensated-FP32 sums (engine count-fp32c), at 20/10 from the
    Dirichlet(1) seed-0 start and at 24/12 from the uniform start.  Per engine:
    iterations/s over `steps` iterations (CUDA events on the engine's stream),
    the q/D pass split, and for count-fp32c the last bound's and rate's
    distance from an FP64 re-evaluation at the same iterate (bdc_bound_error)
    and from the FP64 engine's own bound after the same iterations."""
    import torch

    import bdc_b200
    from bdc_b200 import dist as bdist

    stream = torch.cuda.current_stream()
    out = []
    for n, k, start in [(20, 10, ("dirichlet", 1.0, 0)), (24, 12, ("uniform",))]:
        p0 = bdist.uniform_start(n) if start[0] == "uniform" else bdist.dirichlet_start(n, start[1], start[2])
        iters = max(3, min(args.steps, 40 if n <= 20 else 10))
        row = {"n": n, "k": k, "start": "-".join(map(str, start)), "iters": iters}
        for engine in ("count", "count-fp32c"):
            E = bdc_b200.Engine(n, k, engine=engine)
            E.set_stream(stream.cuda_stream)
            E.set_p(p0)
            E.iterate(3, float("-inf"))
            prof = E.profile(2)
            E.set_p(p0)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st = E.iterate(iters, float("-inf"))
            e1.record(stream)
            torch.cuda.synchronize()
            leg = {"iters_per_s": iters / (e0.elapsed_time(e1) / 1e3), "ms_q": prof["ms_q"], "ms_d": prof["ms_d"],
                   "upper_bound_bits": st["upper_bound"], "rate_bits": st["rate"]}
            if engine == "count-fp32c":
                ub_err, rate_err = E.bound_error()
                leg["bound_err_vs_fp64_reeval_bits"] = ub_err
                leg["rate_err_vs_fp64_reeval_bits"] = rate_err
            row[engine] = leg
            E.close()
        row["fp32c_bound_minus_fp64_engine_bits"] = (row["count-fp32c"]["upper_bound_bits"]
                                                     - row["count"]["upper_bound_bits"])
        row["fp32c_speed_vs_fp64"] = row["count-fp32c"]["iters_per_s"] / row["count"]["iters_per_s"]
        out.append(row)
    return {"precision": out}


GEN_OURS = os.path.join(REPO, "bdc-upper-bounds-gpu_b200", "generate_bit_transition_cache")
GEN_REF = os.path.join(REPO, "oracle", "_ref", "generate_bit_transition_cache")


def _gen_run(exe: str, N: int):
    """One generator process for every cache_{n,k}, n <= N, in an empty
    directory: wall seconds, sha256 over the files (names and bytes), bytes."""
    import hashlib
    import shutil
    d = tempfile.mkdtemp(prefix="bdc_gen_")
    try:
        os.makedirs(os.path.join(d, "transition_counts"))
        t0 = time.perf_counter()
        subprocess.run([exe, str(N)], cwd=d, check=True, stdout=subprocess.DEVNULL, timeout=600)
        sec = time.perf_counter() - t0
        h = hashlib.sha256()
        nbytes = 0
        for f in sorted(os.listdir(os.path.join(d, "transition_counts"))):
            b = open(os.path.join(d, "transition_counts", f), "rb").read()
            nbytes += len(b)
            h.update(f.encode() + b)
        return sec, h.hexdigest(), nbytes
    finally:
        shutil.rmtree(d, ignore_errors=True)


def generator_leg(N: int = 11) -> dict:
    """The reference's CPU cache generator (one host thread, built from its
    sources) beside this repository's GPU generator, both as processes with
    the same argv writing every cache_{n,k} for n <= N; the files must be
    identical."""
    if not os.path.exists(GEN_OURS):
        return {"unavailable": "generate_bit_transition_cache not built"}
    sec, dig, nbytes = _gen_run(GEN_OURS, N)
    row = {"N": N, "bytes": nbytes, "ours_s": sec}
    if os.path.exists(GEN_REF):
        rsec, rdig, _ = _gen_run(GEN_REF, N)
        row.update({"reference_s": rsec, "reference_cores": 1, "identical_files": rdig == dig,
                    "speedup": rsec / sec})
    else:
        row["reference"] = "not built (oracle/Makefile ref)"
    return row


def generator_check(args) -> dict:
    """The cache generator: the reference's CPU program (built from its sources
    into oracle/_ref/, when present) and this repository's GPU one
    (generate_bit_transition_cache, same argv, same files), each run as a
    process in an empty directory, wall clock including the process start (for
    ours the CUDA context too) and the file writes; the files of both must be
    identical.  ours_counts_only_s is the GPU generation of the same tables
    inside this process, copied to host memory, without files.  The reference runs up to N = 12 (its
    time grows about 4x per N: N = 13 takes about a minute), ours up to 13."""
    ours, ref = GEN_OURS, GEN_REF
    run = _gen_run

    # the counts alone, in this process after a warm-up call (no process start,
    # no CUDA context creation, no file writes)
    import bdc_b200
    bdc_b200.generate_cache(4, 2)

    def counts_only(N):
        t0 = time.perf_counter()
        for n in range(N + 1):
            for k in range(n):
                bdc_b200.generate_cache(n, k)
        return time.perf_counter() - t0

    out = []
    for N in (9, 10, 11, 12, 13):
        row = {"N": N}
        sec, dig, nbytes = run(ours, N)
        row.update({"ours_s": sec, "ours_counts_only_s": counts_only(N), "bytes": nbytes})
        if N <= 12 and os.path.exists(ref):
            rsec, rdig, _ = run(ref, N)
            row.update({"reference_s": rsec, "identical_files": rdig == dig, "speedup": rsec / sec})
        out.append(row)
    return {"generator": out, "reference": ref if os.path.exists(ref) else "not built"}


def kernels_only(args) -> None:
    """Engine set-up and `steps` iterations, nothing else: the command that
    the ncu captures under profiles/ run."""
    import bdc_b200
    E = bdc_b200.Engine(args.n, args.k, engine=args.engine, verbose=True)
    E.set_uniform()
    st = E.iterate(args.steps, float("-inf"))
    print(json.dumps({"engine": E.engine, "n": args.n, "k": args.k, "iters": st["iters"],
                      "upper_bound_bits": st["upper_bound"]}))
    E.close()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=24)
    ap.add_argument("--k", type=int, default=12)
    ap.add_argument("--engine", default="auto")
    ap.add_argument("--cpu-sample", type=int, default=20000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--mode", choices=["bench", "kernels", "ttb", "batch", "adjoint", "precision", "gen"],
                    default="bench")
    ap.add_argument("--ttb-budget", type=float, default=15.0,
                    help="device seconds for each of the plain and squarem legs of time-to-bound")
    ap.add_argument("--no-ttb", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the batched time-to-bound and the 26/13 adjoint check in the default line")
    ap.add_argument("--no-ref-cuda", action="store_true",
                    help="skip timing the reference's own CUDA BA (oracle/_ref/ref_harness) on this GPU")
    ap.add_argument("--fd-coords", type=int, default=1024)
    ap.add_argument("--fd-seeds", type=int, default=16)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.mode == "kernels":
        kernels_only(args)
    elif args.mode == "ttb":
        print(json.dumps({"time_to_bound": time_to_bound(args), "n": args.n, "k": args.k}), flush=True)
    elif args.mode == "adjoint":
        print(json.dumps({"adjoint": adjoint_check(args)}), flush=True)
    elif args.mode == "precision":
        print(json.dumps(precision_check(args)), flush=True)
    elif args.mode == "gen":
        print(json.dumps(generator_check(args)), flush=True)
    elif args.mode == "batch":
        res = batched(args)
        if res is not None:
            print(json.dumps({"batched": res}), flush=True)
    elif args.impl == "reference":
        reference_arm(args)
    else:
        ours_arm(args)


if __name__ == "__main__":
    main()
