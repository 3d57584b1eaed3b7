#!/usr/bin/env python3
"""Log-likelihood evaluations per second of the mixed-precision B200 path beside
the plain-FP64 B200 path, at the stated relative error.

Workload (the mixed-precision configuration): N = 102,400 synthetic locations
from the reference generator (jittered 320 x 320 grid, Morton sorted, 16-bit
quantised, srand(0)), observations Z = L e at theta = (1, 0.1, 0.5) with
e = DLARNV(3, {0,0,0,1}) generated on the device, tile 1024.  The mixed form
keeps the diagonal tile and 2 tiles below it in FP64 and stores the other 4,753
tiles in FP32 with split-FP16 tensor-core updates; the plain form is the exact
FP64 path.  One step = one full evaluation (Matern generation, tiled Cholesky,
log-det, triangular solves with one refinement step, assembly) with the
inputs resident in HBM.  The tile storage (22 GB mixed, 42 GB FP64) is far
larger than the 126 MB L2, so no flush is needed.  The relative error is the
mixed log-likelihood against the plain FP64 path at the same N (itself within
1e-10 of the CPU oracle in the tests).

``python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]``
Under torchrun each rank evaluates its own replica (a single evaluation does not
shard): value = evaluations of all ranks / max-over-ranks device time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from exageostatcpp_b200 import replicas as R  # noqa: E402  (pure Python, no GPU needed to import)

N = 102400
DTS = 1024
BAND = 2
THETA = (1.0, 0.1, 0.5)
SEED = 0
METRIC = "loglik evals/s mixed vs plain FP64 on B200 at stated rel. error; p50/p99 ms"
UNIT = "evals/s"
CONFIG = {
    "workload": "MLE log-likelihood evaluation, N=102400 (320x320 jittered grid), 2-D Matern, theta=(1,0.1,0.5), "
                "tile 1024; mixed precision: FP64 diagonal + band of 2 tiles, FP32 off-band tiles with split-FP16 "
                "tcgen05 updates, one refinement step; beside it the plain FP64 path at the same N",
    "n": N, "tile": DTS, "band_tiles": BAND, "theta": list(THETA), "precision": "mixed (value) / fp64 (plain_fp64)",
    "l2": "inputs larger than L2 (22 GB mixed / 42 GB FP64 tile storage vs 126 MB L2); no flush",
}
# The reference's plain-FP64 GPU configuration at N = 40,000: 41,000 points
# generated, 1,000 held out for kriging, tile 960, two true thetas.
C2_TOTAL, C2_MISS, C2_DTS = 41000, 1000, 960
C2_THETAS = ((1.0, 0.03, 1.5), (1.0, 0.05, 0.8))
# The reference's MLE settings (C1 configuration): bounds [0.01, 5]^3, start at
# the lower bounds, ftol_abs 1e-9 (--tolerance=9), at most 100 evaluations.
FIT_LB, FIT_UB, FIT_FTOL, FIT_MAXEVAL = (0.01, 0.01, 0.01), (5.0, 5.0, 5.0), 1e-9, 100
# Fitted theta and MSPE of the mixed form against the plain form at N = 102,400:
# both fits start at the true theta with the same trust radius and budget.
C3_FIT_MAXEVAL, C3_FIT_RHOBEG, C3_MISS = 15, 0.02, 1000
# The batched configuration: 2,048 independent problems, N_i log-uniform in
# [256, 4096], theta_i drawn per problem, one evaluation of all per optimiser step.
C4_B, C4_NMIN, C4_NMAX, C4_SEED = 2048, 256, 4096, 12345
C4_TILES = (128, 192, 256, 320, 384, 512)
# The serving configuration in the default run: two arrival rates, the
# reference's fit budget for fit requests.
SERVE_SECONDS, SERVE_FIT_EVALS = 30.0, 100


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def workload_data(egs):
    """Locations and Z = L e at theta, generated on the device (FP64 path)."""
    x, y = egs.generate_locations(N, SEED)
    gen = egs.Problem(N, DTS)
    gen.set_locations(x, y)
    z = gen.generate_observations(THETA, SEED)
    gen.close()
    return x, y, z


def held_out_data(egs, n_total, dts, theta, n_miss):
    """n_total locations of the reference generator (srand(SEED)), Z = L e at theta
    generated on the device (FP64), then n_miss points held out by the reference's
    random split, which continues the generator's rand() stream
    (PredictionHelpers.cpp:140-168).  Returns (z_obs, x_obs, y_obs, z_miss, x_miss, y_miss)."""
    x, y = egs.generate_locations(n_total, SEED)
    gen = egs.Problem(n_total, dts)
    gen.set_locations(x, y)
    z = gen.generate_observations(theta, SEED)
    gen.close()
    return egs.shuffle_split(z, x, y, n_miss)


def guarded_objective(egs, p):
    """The log-likelihood of problem p as a fit objective.  A theta whose covariance
    is not numerically positive definite scores -1e300 and the search goes on (the
    reference's objective throws there and the fit ends); returns (f, counters)."""
    count = {"evals": 0, "not_positive_definite": 0}

    def f(theta):
        count["evals"] += 1
        try:
            return p.mle_eval(theta)[0]
        except egs.NotPositiveDefinite:
            count["not_positive_definite"] += 1
            return -1e300
    return f, count


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


class ClockSampler:
    """nvidia-smi samples (every 200 ms) of the SM clock and throttle reasons."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, bus_id: str | None):
        self.proc = None
        self.bus_id = bus_id

    def start(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if self.bus_id:
            cmd += ["-i", self.bus_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for name, v in zip(names, parts[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def fp64_dgemm_peak_tflops(torch) -> float:
    """cuBLAS DGEMM throughput on this GPU (the FP64 tensor roofline), best of 5 at 8192^3."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        a @ b
    torch.cuda.synchronize()
    best = 1e30
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(5):
        e0.record()
        a @ b
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def small_problem_rate(egs, torch, steps: int = 200):
    """Evaluations/s of the reference's N = 1,600, tile 320 configuration (CUDA-graph replay)."""
    x, y = egs.generate_locations(1600, 0)
    p = egs.Problem(1600, 320)
    p.set_locations(x, y)
    p.generate_observations((1.0, 0.1, 0.5), 0)
    for _ in range(5):
        p.mle_eval((1.0, 0.1, 0.5))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        p.mle_eval((1.0, 0.1, 0.5))
    dt = time.perf_counter() - t0
    p.close()
    return {"config": "N=1600, tile 320, theta=(1,0.1,0.5), one GPU, host-timed incl. result read-back",
            "evals_per_s": steps / dt, "ms_per_eval": 1e3 * dt / steps}


def cpu_sample(x, y, z, target_s: float = 12.0):
    """Time the CPU restatement on a bounded sample; returns (evals/s scaled to N, info)."""
    from oracle import cpu_baseline as C
    n_target = len(z)
    ns = 6000
    ll, st = C.timed_eval(x[:ns], y[:ns], z[:ns], THETA)
    est = sum(st.values())
    grow = (target_s / max(est, 1e-3)) ** (1.0 / 3.0)
    ns2 = int(min(20000, max(6000, ns * grow)) // 64 * 64)
    if ns2 > ns:
        ns = ns2
        ll, st = C.timed_eval(x[:ns], y[:ns], z[:ns], THETA)
    value = C.scaled_evals_per_s(st, ns, n_target)
    return value, {
        "cores": C.threads(), "n_sample": ns, "stage_s": {k: round(v, 4) for k, v in st.items()},
        "sample": f"one full FP64 evaluation at N={ns} (first {ns} of the workload's points, theta={THETA}); "
                  f"generation and solve scaled by (N/{ns})^2, potrf by (N/{ns})^3 to N={n_target}"}


def run_reference(args):
    """The reference's FP64 path on the host cores (the oracle's restatement: Matern
    generation in C on all threads, blocked Cholesky and solves on OpenBLAS).

    Measured in this run: one full evaluation at N = 102,400 (84 GB of host
    memory) and one at the N = 40,000 configuration.  The K timed steps are
    bounded samples (one evaluation of the first N_s points each), projected to
    N = 102,400 by the stages' n^2 / n^3 cost model and multiplied by the ratio
    of the measured full-size evaluation to the projection of the warm-up
    samples, so that the reported rate rests on the measured full-size time."""
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import cpu_baseline as C
    from oracle import oracle as O
    # Same locations as the B200 arm, produced on the host by the oracle's
    # generator; observations from DLARNV (the cost does not depend on them).
    t0 = time.perf_counter()
    x, y = O.generate_locations(N, O.GlibcRand(SEED))
    full = None
    if not args.no_full_cpu:
        zf = O.dlarnv_normal(SEED, N)
        ll_full, st_full = C.timed_eval(x, y, zf, THETA)
        del zf
        full = {"n": N, "seconds": sum(st_full.values()), "stage_s": {k: round(v, 3) for k, v in st_full.items()},
                "loglik": ll_full}
    # the N = 40,000 configuration: the training split of 41,000 points
    rng = O.GlibcRand(SEED)
    x2, y2 = O.generate_locations(C2_TOTAL, rng)
    z2 = O.dlarnv_normal(SEED, C2_TOTAL)
    z2o, x2o, y2o, _, _, _ = O.shuffle_split(z2, x2, y2, C2_MISS, rng)
    _, st_c2 = C.timed_eval(x2o, y2o, z2o, C2_THETAS[1])
    c2 = {"n": len(z2o), "theta": list(C2_THETAS[1]), "seconds": sum(st_c2.values()),
          "evals_per_s": 1.0 / sum(st_c2.values()), "stage_s": {k: round(v, 3) for k, v in st_c2.items()}}
    # bounded samples for the timed steps
    ns = 6000
    z = O.dlarnv_normal(SEED, ns)
    _, st = C.timed_eval(x[:ns], y[:ns], z, THETA)
    per_step = 3.0
    grow = (per_step / max(sum(st.values()), 1e-3)) ** (1.0 / 3.0)
    ns = int(min(16000, max(4000, ns * grow)) // 64 * 64)
    z = O.dlarnv_normal(SEED, ns)
    a = np.zeros((ns, ns), order="F")
    projected = []
    for _ in range(args.warmup):
        _, st = C.timed_eval(x[:ns], y[:ns], z, THETA, a)
        projected.append(1.0 / C.scaled_evals_per_s(st, ns, N))
    calib = full["seconds"] / statistics.mean(projected) if full else 1.0
    scaled = []
    lat = []
    for _ in range(args.steps):
        _, st = C.timed_eval(x[:ns], y[:ns], z, THETA, a)
        scaled.append(calib / C.scaled_evals_per_s(st, ns, N))
        lat.append(sum(st.values()))
    total = sum(scaled)
    value = args.steps / total
    how = (f"each step one full FP64 evaluation at N={ns} on all host threads (Matern in C/pthreads, blocked "
           f"Cholesky and solves on OpenBLAS), projected to N={N} by n^2 (generation, solve) and n^3 (potrf)")
    if full:
        how += (f" and calibrated by x{calib:.3f}, the ratio of the full N={N} evaluation measured in this run "
                f"({full['seconds']:.1f} s) to the projection of the warm-up samples")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference generator semantics)",
        "config": CONFIG,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": C.threads(), "kind": "port", "sample": how,
                         "measured_full_n": full, "calibration": calib, "measured_c2": c2},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "p50_ms": 1e3 * statistics.median(scaled), "p99_ms": 1e3 * float(np.percentile(scaled, 99)),
        "sample_step_s_p50": statistics.median(lat), "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)
    return 0


def warm_profiled(p, theta):
    """Last warm-up step: turn per-stage timing on and run one evaluation, which
    captures the replayed graph with its timing events outside the timed region;
    then start the stage totals afresh."""
    p.set_profiling(True)
    p.mle_eval(theta)
    p.set_profiling(True)


def timed_evals(torch, p, stream, theta, steps, dist=None):
    """Device time (ms, max over ranks) of `steps` evaluations, host latencies (ms) and the last result."""
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lat = []
    e0.record(stream)
    for _ in range(steps):
        t = time.perf_counter()
        r = p.mle_eval(theta)
        lat.append(1e3 * (time.perf_counter() - t))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = R.max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    return ms, lat, r


def c2_leg(egs, torch, steps, peak):
    """The reference's plain-FP64 GPU configuration, end to end, for both true thetas:
    41,000 points (a 203-wide jittered grid, srand(0)), 1,000 held out by the
    reference's split, tile 960; device-timed evaluations at the true theta with
    the trailing-update roofline, a full fit with the reference's MLE settings
    (BOBYQA from the lower bounds, ftol_abs 1e-9, at most 100 evaluations), then
    kriging of the 1,000 held-out points at the fitted theta and MSPE against the
    truth (LinearAlgebraMethods.cpp:527-577)."""
    import numpy as np
    out = []
    for theta in C2_THETAS:
        zo, xo, yo, za, xm, ym = held_out_data(egs, C2_TOTAL, C2_DTS, theta, C2_MISS)
        stream = torch.cuda.Stream()
        p = egs.Problem(len(zo), C2_DTS)
        p.set_stream(stream.cuda_stream)
        p.set_locations(xo, yo)
        p.set_observations(zo)
        for _ in range(2):
            p.mle_eval(theta)
        warm_profiled(p, theta)
        ms, _, r = timed_evals(torch, p, stream, theta, steps)
        st_ms, st_fl, _ = p.stage_stats()
        p.set_profiling(False)
        up = egs.STAGES.index("update")
        ach = st_fl[up] / (st_ms[up] * 1e-3) / 1e12
        f, count = guarded_objective(egs, p)
        t0 = time.perf_counter()
        th, fb, ne = egs.bobyqa_maximize(f, FIT_LB, FIT_LB, FIT_UB, FIT_FTOL, FIT_MAXEVAL)
        fit_s = time.perf_counter() - t0
        zm = p.predict(th, xm, ym)
        zt = p.predict(theta, xm, ym)
        p.close()
        out.append({
            "theta_true": list(theta), "n": len(zo), "n_miss": len(za), "tile": C2_DTS,
            "evals_per_s": steps / (ms * 1e-3), "ms_per_eval": ms / steps, "loglik_at_true": r[0],
            "logdet_at_true": r[1], "dot_at_true": r[2],
            "trailing_update_tflops": ach, "trailing_update_frac_of_dgemm": ach / peak,
            "fit": {"theta": th.tolist(), "loglik": fb, "evals": ne, "seconds": fit_s,
                    "evals_per_s": count["evals"] / fit_s, "not_positive_definite": count["not_positive_definite"],
                    "settings": "BOBYQA, bounds [0.01,5]^3, start at the lower bounds, ftol_abs 1e-9, "
                                "maxeval 100"},
            "mspe_at_fit": float(np.mean((za - zm) ** 2)), "mspe_at_true": float(np.mean((za - zt) ** 2)),
        })
    return {"config": "plain FP64, N=40000 (41000 generated on a 203-wide jittered grid, srand(0); 1000 held out "
                      "by the reference's rand() split), tile 960", "thetas": out}


def c4_problems(egs):
    """The batched configuration's problems: seed_i = i (the reference generator's
    srand and DLARNV seeds), N_i = round(exp(U[ln 256, ln 4096])), sigma^2 ~ U[0.5, 2],
    beta ~ U[0.02, 0.3], nu ~ U[0.3, 2.5] from one seeded host generator; jittered-grid
    locations; observations are DLARNV N(0, 1) draws (an evaluation's cost does
    not depend on their values).  Returns (sizes, x, y, z concatenated, theta (B, 3))."""
    import numpy as np
    rng = np.random.default_rng(C4_SEED)
    sizes = np.rint(np.exp(rng.uniform(math.log(C4_NMIN), math.log(C4_NMAX), C4_B))).astype(np.int32)
    theta = np.column_stack([rng.uniform(0.5, 2.0, C4_B), rng.uniform(0.02, 0.3, C4_B),
                             rng.uniform(0.3, 2.5, C4_B)])
    xs, ys, zs = [], [], []
    for i, n in enumerate(sizes):
        x, y = egs.generate_locations(int(n), i)
        xs.append(x)
        ys.append(y)
        zs.append(egs.dlarnv_normal(i % 4096, int(n)))
    return sizes, np.concatenate(xs), np.concatenate(ys), np.concatenate(zs), theta


def c4_leg(egs, torch, steps):
    """Batched evaluations of the 2,048-problem configuration: the tile size chosen
    by the autotuner (one timed graph replay per candidate), then `steps` timed
    replays (CUDA events), against the same problems evaluated one at a time on
    the plain FP64 path (each problem's own graph replayed, the host waiting for
    every result as a one-problem-per-call caller does).  Problems whose
    covariance is not numerically positive definite (smooth, long-range
    draws) are evaluated all the same and counted."""
    import numpy as np
    sizes, x, y, z, theta = c4_problems(egs)
    t0 = time.perf_counter()
    upper, tiles, tune_ms = egs.batch_set_autotune(sizes, x, y, z, theta, candidates=C4_TILES, max_classes=3)
    tune_s = time.perf_counter() - t0
    ts1, one_class_ms = egs.batch_autotune(sizes, x, y, z, theta, candidates=C4_TILES)
    b = egs.BatchSet(sizes, x, y, z, upper_n=upper, dts=tiles)
    for _ in range(3):
        ll, st = b.eval(theta)
    info = b.info()
    # every step waits for its results (the optimiser needs them), so the host
    # clock around the steps is the step time
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        ll, st = b.eval(theta)
    host_s = time.perf_counter() - t0
    b.close()
    batch_evals_per_s = C4_B * steps / (host_s)
    # one problem at a time, same problems and thetas, FP64, graph replay
    offs = np.concatenate([[0], np.cumsum(sizes)])
    single_s = 0.0
    single_ll = np.empty(C4_B)
    for i, n in enumerate(sizes):
        p = egs.Problem(int(n), next(t for u, t in zip(info["upper_n"], info["ts"]) if n <= u))
        p.set_locations(x[offs[i]:offs[i + 1]], y[offs[i]:offs[i + 1]])
        p.set_observations(z[offs[i]:offs[i + 1]])
        for _ in range(2):
            try:
                p.mle_eval(theta[i])
            except egs.NotPositiveDefinite:
                pass
        t1 = time.perf_counter()
        try:
            single_ll[i] = p.mle_eval(theta[i])[0]
        except egs.NotPositiveDefinite:
            single_ll[i] = np.nan
        single_s += time.perf_counter() - t1
        p.close()
    ok = st == 0
    agree = np.abs(ll[ok] - single_ll[ok]) / np.abs(single_ll[ok])
    # whether the mixed-precision form could pay off at these sizes: one problem
    # of N points evaluated in both forms (tile 256, FP64 band of 2 tiles)
    mixed_vs_plain = []
    for n in (1024, 2048, 4096):
        xx, yy = egs.generate_locations(n, 0)
        zz = egs.dlarnv_normal(0, n)
        row = {"n": n}
        for label, prec in (("plain_ms", egs.EGS_PRECISION_DOUBLE), ("mixed_ms", egs.EGS_PRECISION_MIXED)):
            p = egs.Problem(n, 256)
            if prec == egs.EGS_PRECISION_MIXED:
                p.set_precision(prec, 2)
            p.set_locations(xx, yy)
            p.set_observations(zz)
            for _ in range(3):
                p.mle_eval((1.0, 0.1, 0.5))
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            for _ in range(20):
                p.mle_eval((1.0, 0.1, 0.5))
            row[label] = 1e3 * (time.perf_counter() - t1) / 20
            p.close()
        mixed_vs_plain.append(row)
    flops = float(np.sum(sizes.astype(np.float64) ** 3 / 3.0))
    return {"config": f"{C4_B} problems, N_i log-uniform in [{C4_NMIN}, {C4_NMAX}] (sum {int(sizes.sum())}), "
                      "theta_i: sigma2 ~ U[0.5,2], beta ~ U[0.02,0.3], nu ~ U[0.3,2.5]; plain FP64",
            "schedule": {"classes": info["classes"], "upper_n": info["upper_n"], "tiles": info["ts"]},
            "autotune": {"candidates": list(C4_TILES), "max_classes": 3, "best_ms_per_eval": tune_ms,
                         "seconds": tune_s, "one_class_tile": ts1, "one_class_ms_per_eval": one_class_ms},
            "evals_per_s": batch_evals_per_s, "ms_per_step": 1e3 * host_s / steps, "steps": steps,
            "not_positive_definite": int((~ok).sum()),
            "potrf_tflops": flops / (host_s / steps) / 1e12,
            "one_at_a_time_evals_per_s": C4_B / single_s, "one_at_a_time_s": single_s,
            "speedup_vs_one_at_a_time": batch_evals_per_s / (C4_B / single_s),
            "max_rel_diff_vs_one_at_a_time": float(agree.max()) if agree.size else None,
            "single_problem_mixed_vs_plain": mixed_vs_plain}


def c3_fit_leg(egs):
    """Fitted theta and MSPE of the mixed form against the plain FP64 form at
    N = 102,400: N + 1,000 points generated (Z = L e at the true theta, FP64), 1,000
    held out by the reference's split, the 102,400 others fitted by BOBYQA in each
    form from the true theta (trust radius 0.02, the same budget of evaluations,
    bounds [0.01, 5]^3, ftol_abs 1e-9), then kriging of the held-out points at each
    form's fitted theta with its own factorisation (mixed: FP32 off-band storage
    and one refinement step).  The plain form also evaluates its likelihood at the
    mixed form's fitted theta: how much likelihood the mixed fit gives up."""
    import numpy as np
    zo, xo, yo, za, xm, ym = held_out_data(egs, N + C3_MISS, DTS, THETA, C3_MISS)
    res = {}
    for label in ("mixed", "plain"):
        p = egs.Problem(len(zo), DTS)
        if label == "mixed":
            p.set_precision(egs.EGS_PRECISION_MIXED, BAND)
        p.set_locations(xo, yo)
        p.set_observations(zo)
        f, count = guarded_objective(egs, p)
        t0 = time.perf_counter()
        th, fb, ne = egs.bobyqa_maximize(f, THETA, FIT_LB, FIT_UB, FIT_FTOL, C3_FIT_MAXEVAL, rhobeg=C3_FIT_RHOBEG)
        fit_s = time.perf_counter() - t0
        zm = p.predict(th, xm, ym)
        res[label] = {"theta": th.tolist(), "loglik": fb, "evals": ne, "seconds": fit_s,
                      "not_positive_definite": count["not_positive_definite"],
                      "mspe": float(np.mean((za - zm) ** 2)), "z_miss": zm}
        if label == "plain":
            res["plain_loglik_at_mixed_theta"] = p.mle_eval(res["mixed"]["theta"])[0]
        p.close()
    tm, tp = np.array(res["mixed"]["theta"]), np.array(res["plain"]["theta"])
    zm_m, zm_p = res["mixed"].pop("z_miss"), res["plain"].pop("z_miss")
    theta = {"mixed": res["mixed"], "plain": res["plain"], "abs_diff": np.abs(tm - tp).tolist(),
             "rel_diff": (np.abs(tm - tp) / np.abs(tp)).tolist(),
             "plain_loglik_loss_at_mixed_theta": res["plain"]["loglik"] - res["plain_loglik_at_mixed_theta"],
             "settings": f"N={len(zo)} of {N + C3_MISS} generated ({C3_MISS} held out), BOBYQA from the true theta, "
                         f"rhobeg {C3_FIT_RHOBEG}, maxeval {C3_FIT_MAXEVAL}, bounds [0.01,5]^3, ftol_abs 1e-9, "
                         "both forms"}
    mspe = {"mixed": res["mixed"]["mspe"], "plain": res["plain"]["mspe"],
            "rel_diff": abs(res["mixed"]["mspe"] - res["plain"]["mspe"]) / res["plain"]["mspe"],
            "prediction_max_rel_diff": float(np.abs(zm_m - zm_p).max() / np.abs(zm_p).max()),
            "note": "each form krieges at its own fitted theta with its own factorisation"}
    return theta, mspe


def run_serving(args):
    """``--workload serving``: the sweep alone, one JSON line per (form, rate) and a summary."""
    import torch
    import exageostatcpp_b200 as egs
    torch.cuda.set_device(0)
    lines = serving_sweep(egs, args.serve_rates, args.serve_seconds, args.serve_slots, args.serve_fit_evals,
                          verbose=True)
    print(json.dumps({"metric": METRIC, "workload": "serving", "unit": UNIT, "slots": args.serve_slots,
                      "hbm_budget_gb": 160, "fit_max_evals": args.serve_fit_evals, "sweep": lines}), flush=True)
    return 0


def serving_sweep(egs, rates, seconds, slots, fit_evals, verbose=False):
    """Open-loop Poisson request stream through the serving loop, rate swept.

    Mix: 35% log-likelihood, 35% fit (BOBYQA, at most --serve-fit-evals
    evaluations), 30% predict (500 targets); N log-uniform in [1,000, 60,000]
    on jittered grids, theta drawn as sigma^2 ~ U[0.5, 2], beta ~ U[0.02, 0.3],
    nu ~ U[0.3, 2.5]; observations are i.i.d. N(0, 1) (the cost does not depend
    on their values).  HBM admission budget 160 GB.  Reports p50/p99 latency
    (submission to completion) and evaluations/s per rate, for the plain and the
    mixed form (FP64 band of 2 tiles)."""
    import numpy as np
    rng = np.random.default_rng(12345)
    pool = []
    for i in range(24):
        n = int(round(math.exp(rng.uniform(math.log(1000), math.log(60000)))))
        x, y = egs.generate_locations(n, i % 4096)
        z = rng.standard_normal(n)
        pool.append((x, y, z))
    xm_all, ym_all = rng.random(500), rng.random(500)
    lines = []
    for rate in rates:
        # one arrival sequence per rate, replayed for both forms
        g = np.random.default_rng(int(rate * 1000) + 7)
        arr = []
        t = 0.0
        while True:
            t += g.exponential(1.0 / rate)
            if t > seconds:
                break
            arr.append(t)
        picks = []
        for a in arr:
            u = g.random()
            kind = egs.EGS_REQ_LOGLIK if u < 0.35 else (egs.EGS_REQ_FIT if u < 0.70 else egs.EGS_REQ_PREDICT)
            theta = (g.uniform(0.5, 2.0), g.uniform(0.02, 0.3), g.uniform(0.3, 2.5))
            picks.append((a, int(g.integers(len(pool))), kind, theta))
        for precision, label in ((egs.EGS_PRECISION_DOUBLE, "plain"), (egs.EGS_PRECISION_MIXED, "mixed")):
            reqs = []
            for a, idx, kind, theta in picks:
                x, y, z = pool[idx]
                dts = 512 if len(z) < 8000 else 1024
                r = dict(kind=kind, x=x, y=y, z=z, dts=dts, theta=theta, precision=precision,
                         band_tiles=2 if precision == egs.EGS_PRECISION_MIXED else 0,
                         max_evals=fit_evals, ftol_abs=1e-9)
                if kind == egs.EGS_REQ_PREDICT:
                    r["x_miss"], r["y_miss"] = xm_all, ym_all
                reqs.append((a, r))
            with egs.Server(hbm_budget=160 * 10**9, max_active=slots) as srv:
                t0 = time.perf_counter()
                tickets = []
                for a, r in reqs:
                    d = a - (time.perf_counter() - t0)
                    if d > 0:
                        time.sleep(d)
                    tickets.append(srv.submit(**r))
                res = [srv.wait(tk)[0] for tk in tickets]
                span = time.perf_counter() - t0
                st = srv.stats()
            lat = np.array([r.latency_ms for r in res])
            kinds = {egs.EGS_REQ_LOGLIK: "loglik", egs.EGS_REQ_FIT: "fit", egs.EGS_REQ_PREDICT: "predict"}
            per = {}
            for k, name in kinds.items():
                lk = np.array([r.latency_ms for r in res if r.kind == k])
                if len(lk):
                    per[name] = {"n": int(len(lk)), "p50_ms": float(np.percentile(lk, 50)),
                                 "p99_ms": float(np.percentile(lk, 99))}
            lines.append({"form": label, "rate_per_s": rate, "requests": len(res),
                          "failed": int(sum(r.status != 0 for r in res)),
                          "failed_not_positive_definite": int(sum(r.status > 0 for r in res)),
                          "answered_in_fp64": int(sum(r.precision_used != precision for r in res)),
                          "fp64_predicted": int(sum(r.fp64_reason == egs.EGS_FP64_REASON_PREDICTED for r in res)),
                          "fp64_after_failure": int(sum(r.fp64_reason == egs.EGS_FP64_REASON_AFTER_FAILURE
                                                        for r in res)),
                          "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                          "evals_per_s": st["evals"] / span, "span_s": span, "per_kind": per,
                          "peak_active": st["peak_active"], "peak_reserved_gb": st["peak_reserved"] / 1e9})
            if verbose:
                print(json.dumps(lines[-1]), flush=True)
    return lines


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-full-cpu", action="store_true",
                    help="reference arm: skip the measured full-size CPU evaluation (84 GB of host memory)")
    ap.add_argument("--no-batched", action="store_true", help="skip the 2,048-problem batched leg")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving sweep of the default run")
    ap.add_argument("--no-fits", action="store_true",
                    help="skip the fitted-theta / MSPE legs (N=102,400 mixed vs plain fits, N=40,000 fits)")
    ap.add_argument("--plain-steps", type=int, default=2, help="timed plain-FP64 evaluations at N=102400")
    ap.add_argument("--profile-eval", action="store_true",
                    help="one mixed evaluation between cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--profile-n", type=int, default=0,
                    help="with --profile-eval: evaluate this many points of a jittered grid with DLARNV "
                         "observations instead of the full workload (small ncu captures)")
    ap.add_argument("--profile-plain", action="store_true", help="with --profile-eval: the plain FP64 path")
    ap.add_argument("--profile-batched", type=int, default=0,
                    help="the first B problems of the batched configuration in one size class at --profile-tile: "
                         "six evaluations (direct launches, graph capture, replays) for ncu launch lists")
    ap.add_argument("--profile-tile", type=int, default=320)
    ap.add_argument("--workload", default="eval", choices=["eval", "serving"])
    ap.add_argument("--serve-rates", type=float, nargs="+", default=[0.25, 0.5, 1.0])
    ap.add_argument("--serve-seconds", type=float, default=30.0)
    ap.add_argument("--serve-slots", type=int, default=6)
    ap.add_argument("--serve-fit-evals", type=int, default=SERVE_FIT_EVALS)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serving":
        return run_serving(args)

    import numpy as np
    import torch
    import exageostatcpp_b200 as egs

    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    props = torch.cuda.get_device_properties(dev)
    bus = None
    try:
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
    except AttributeError:
        pass

    if args.profile_batched:
        sizes, x, y, z, theta = c4_problems(egs)
        nb = int(min(args.profile_batched, C4_B))
        npts = int(sizes[:nb].sum())
        b = egs.Batch(sizes[:nb], x[:npts], y[:npts], z[:npts], dts=args.profile_tile)
        t0 = time.perf_counter()
        for _ in range(6):
            b.eval(theta[:nb])
        print(json.dumps({"problems": nb, "tile": args.profile_tile, "ms_per_step_incl_capture":
                          1e3 * (time.perf_counter() - t0) / 6, "info": b.info()}), flush=True)
        b.close()
        return 0

    if args.profile_eval:
        if args.profile_n:
            x, y = egs.generate_locations(args.profile_n, SEED)
            z = egs.dlarnv_normal(SEED, args.profile_n)
        else:
            x, y, z = workload_data(egs)
        p = egs.Problem(len(z), DTS)
        if not args.profile_plain:
            p.set_precision(egs.EGS_PRECISION_MIXED, BAND)
        p.set_locations(x, y)
        p.set_observations(z)
        p.mle_eval(THETA)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        p.mle_eval(THETA)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        p.close()
        return 0

    peaks = load_peaks()
    fp64_peak = fp64_dgemm_peak_tflops(torch)
    x, y, z = workload_data(egs)

    # --- mixed precision: the headline -------------------------------------------------
    stream = torch.cuda.Stream()
    q = egs.Problem(N, DTS)
    q.set_precision(egs.EGS_PRECISION_MIXED, BAND)
    q.set_stream(stream.cuda_stream)
    q.set_locations(x, y)
    q.set_observations(z)
    for _ in range(args.warmup - 1):
        q.mle_eval(THETA)
    warm_profiled(q, THETA)
    clocks = ClockSampler(bus)
    clocks.start()
    ms, lat, (ll, logdet, dot) = timed_evals(torch, q, stream, THETA, args.steps, dist)
    clk = clocks.stop()
    stage_ms, stage_flops, stage_launches = q.stage_stats()
    q.set_profiling(False)
    value = world * args.steps / (ms * 1e-3)

    # end to end through the C ABI with host buffers: locations and observations
    # uploaded from pinned host memory every step, the result read back
    pin = [torch.from_numpy(a).pin_memory() for a in (x, y, z)]
    xh, yh, zh = (t.numpy() for t in pin)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        q.set_locations(xh, yh)
        q.set_observations(zh)
        ll_e2e = q.mle_eval(THETA)[0]
    e2e_s = R.max_over_ranks(time.perf_counter() - t0, dist, "cuda")
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * N * 8 + 64,
           "d2h_bytes_per_step": 4 * 8 + 8,
           "api": "egs_problem_set_locations + egs_problem_set_observations + egs_mle_eval "
                  "(C ABI, pinned host buffers, mixed precision)"}
    q.close()

    # --- plain FP64 at the same N: speed and the accuracy reference ----------------------
    ps = torch.cuda.Stream()
    p = egs.Problem(N, DTS)
    p.set_stream(ps.cuda_stream)
    p.set_locations(x, y)
    p.set_observations(z)
    p.mle_eval(THETA)
    warm_profiled(p, THETA)
    pms, plat, (pll, plogdet, pdot) = timed_evals(torch, p, ps, THETA, args.plain_steps, dist)
    p_ms, p_fl, p_ln = p.stage_stats()
    p.close()
    plain_value = world * args.plain_steps / (pms * 1e-3)
    up = egs.STAGES.index("update")
    plain_update = p_fl[up] / (p_ms[up] * 1e-3) / 1e12
    plain = {"value": plain_value, "unit": UNIT, "ms_per_eval": pms / args.plain_steps,
             "p50_ms": statistics.median(plat), "loglik": pll, "logdet": plogdet, "dot": pdot,
             "trailing_update_tflops": plain_update, "trailing_update_frac_of_dgemm": plain_update / fp64_peak,
             "stages_ms_per_eval": {s: float(p_ms[i]) / args.plain_steps for i, s in enumerate(egs.STAGES)},
             "steps": args.plain_steps, "warmup": 2}
    rel = {"loglik": abs(ll - pll) / abs(pll), "logdet": abs(logdet - plogdet) / abs(plogdet),
           "dot": abs(dot - pdot) / abs(pdot), "against": "plain FP64 B200 path at the same N"}

    # --- rooflines of the update kernels (CUDA events around every launch) ---------------
    # DRAM bytes (read + write) per algorithmic flop of each kernel, from one ncu
    # capture of each at N = 16,384: the split kernel moved 789,244,160 B for 78
    # target tiles of 2 * 1024^3 flops; the Ozaki kernel 654,302,464 B for the band
    # update of step 0, 7.410e10 FP64-equivalent flops.
    # Both kernels' traffic grows with their target tiles, so a launch's traffic
    # is this ratio times its flops.
    split_bytes_per_flop = 789244160.0 / (78 * 2.0 * 1024 ** 3)
    ozaki_bytes_per_flop = 654302464.0 / 7.410e10
    traffic_note = ("DRAM read + write bytes per flop from one ncu capture at N=16384, times this launch's "
                    "algorithmic flops")
    lo = egs.STAGES.index("update_low")
    bf16_peak = peaks.get("bf16_tflops_sustained") or 1386.0
    roofs = []
    if stage_ms[lo] > 0:
        a = stage_flops[lo] / (stage_ms[lo] * 1e-3) / 1e12
        n_l = int(stage_launches[lo])
        roofs.append({"bound": "tensor", "kernel": "split_gemm_kernel (off-band C -= P_i P_j^T, split-FP16 tcgen05, "
                                                   "FP32-accurate)",
                      "achieved": a, "peak": bf16_peak, "unit": "TFLOP/s", "frac": a / bf16_peak,
                      "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)",
                      "executed_tflops": 3.0 * a, "frac_executed": 3.0 * a / bf16_peak,
                      "note": "achieved counts the algorithmic 2*ts^3 flops per target tile; the kernel executes "
                              "three FP16 products per tile (hi*hi, hi*lo, lo*hi)",
                      "traffic": split_bytes_per_flop * stage_flops[lo] / max(n_l, 1), "traffic_unit": "B",
                      "traffic_source": traffic_note,
                      "launches": n_l, "ms_per_eval": float(stage_ms[lo]) / args.steps,
                      "flops_per_launch": stage_flops[lo] / max(n_l, 1)})
    if stage_ms[up] > 0:
        a = stage_flops[up] / (stage_ms[up] * 1e-3) / 1e12
        n_u = int(stage_launches[up])
        int8_peak = 2.0 * bf16_peak
        roofs.append({"bound": "tensor",
                      "kernel": "ozaki_band_kernel (FP64-class band update: 7 signed 7-bit slices per operand, "
                                "exact int32 products on tcgen05 kind::i8, ten MMAs of N <= 256 per K step)",
                      "achieved": a, "peak": fp64_peak, "unit": "TFLOP/s", "frac": a / fp64_peak,
                      "peak_source": "FP64-equivalent flops against cuBLAS DGEMM 8192^3 measured in this run "
                                     "(MEASURED_PEAKS.json has no FP64 entry)",
                      "executed_int8_tops": 28.0 * a, "frac_executed_of_int8": 28.0 * a / int8_peak,
                      "int8_peak_source": "2x MEASURED_PEAKS.json bf16_tflops_sustained (the int8 rate is twice "
                                          "the bf16 rate on B200)",
                      "traffic": ozaki_bytes_per_flop * stage_flops[up] / max(n_u, 1), "traffic_unit": "B",
                      "traffic_source": traffic_note,
                      "launches": n_u, "ms_per_eval": float(stage_ms[up]) / args.steps,
                      "flops_per_launch": stage_flops[up] / max(n_u, 1)})
    roofs.sort(key=lambda r: -r["ms_per_eval"])
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f16/f32/f64 (mixed)",
        "data": "synthetic (reference generator semantics, generated on device)",
        "config": dict(CONFIG, parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "loglik": ll, "loglik_e2e": ll_e2e, "logdet": logdet, "dot": dot,
        "p50_ms": statistics.median(lat), "p99_ms": float(np.percentile(lat, 99)),
        "plain_fp64": plain, "speedup_vs_plain": value / plain_value, "rel_error": rel,
        "stages_ms_per_eval": {s: float(stage_ms[i]) / args.steps for i, s in enumerate(egs.STAGES)},
        "roofline": roofs[0] if roofs else None, "roofline_other": roofs[1:],
        "e2e": e2e,
        "gpu_launches": int(stage_launches.sum()),
        "clocks": clk,
    }
    if world == 1 and not args.no_fits:
        rel["theta"], rel["mspe"] = c3_fit_leg(egs)
        line["c2"] = c2_leg(egs, torch, 3, fp64_peak)
    if world == 1 and not args.no_batched:
        line["batched"] = c4_leg(egs, torch, 5)
    if world == 1 and not args.no_serving:
        rates = (0.15, 0.3)
        line["serving"] = {
            "config": f"open-loop Poisson arrivals for {SERVE_SECONDS:.0f} s per rate, 35% log-likelihood, 35% fit "
                      f"(BOBYQA, at most {SERVE_FIT_EVALS} evaluations, ftol_abs 1e-9: the reference's MLE budget), "
                      "30% predict (500 targets); N log-uniform in [1000, 60000]; theta as in the batched "
                      "configuration; 160 GB admission budget; 6 slots; observations i.i.d. N(0,1)",
            "sweep": serving_sweep(egs, rates, SERVE_SECONDS, 6, SERVE_FIT_EVALS)}
    line["small_n"] = small_problem_rate(egs, torch)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, info = cpu_sample(x, y, z)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "port",
                                "sample": info["sample"], "stage_s": info["stage_s"]}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
