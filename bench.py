#!/usr/bin/env python3
"""Log-likelihood evaluations per second of the plain-FP64 B200 path.

Workload (the reference's N = 40,000 plain-FP64 configuration): 41,000 synthetic
locations from the reference generator (jittered 203 x 203 grid, Morton sorted,
16-bit quantised, srand(0)), observations Z = L e at theta_true = (1, 0.05, 0.8)
with e = DLARNV(3, {0,0,0,1}), 1,000 points held out at random, and the
log-likelihood of the remaining N = 40,000 evaluated at theta_true with tile 960.
One step = one full evaluation (Matern generation, tiled Cholesky, log-det,
triangular solve, dot, assembly) with the inputs resident in HBM.  The tile
storage is 6.6 GB, far larger than the 126 MB L2, so no flush is needed.

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

N_TOTAL = 41000
N_MISS = 1000
DTS = 960
THETA = (1.0, 0.05, 0.8)
SEED = 0
METRIC = "loglik evals/s (plain FP64, N=40000 Matern, tile 960)"
UNIT = "evals/s"
CONFIG = {
    "workload": "MLE log-likelihood evaluation, N=40000 (41000 generated, 1000 held out), 2-D Matern, "
                "theta=(1,0.05,0.8), tile 960, plain FP64",
    "n": N_TOTAL - N_MISS, "tile": DTS, "theta": list(THETA), "precision": "fp64",
    "l2": "inputs larger than L2 (6.6 GB tile storage vs 126 MB L2); no flush",
}
# DRAM bytes per updated C element of the trailing-update kernel, from one ncu
# capture of a full trailing update (N = 8,000, tile 960: 571 MB for 1,830
# 128 x 128 blocks; profiles/dgemm_update_kernel_n8000.md).  The per-launch
# traffic of this workload is that figure times each launch's block count.
UPDATE_DRAM_BYTES_PER_C_ELEMENT = 571.28e6 / (1830 * 128 * 128)


def update_traffic_per_launch(n: int, ts: int) -> float:
    """Mean DRAM bytes of one trailing-update launch at (n, ts), scaled from the capture."""
    nt = -(-n // ts)
    per = []
    for k in range(nt - 1):
        mb = -(-((nt - k - 1) * ts) // 128)
        per.append(mb * (mb + 1) // 2 * 128 * 128 * UPDATE_DRAM_BYTES_PER_C_ELEMENT)
    return sum(per) / max(len(per), 1)


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def workload_data(egs):
    """Locations, Z (generated on the device), and the 40,000-point training split."""
    import numpy as np
    x, y = egs.generate_locations(N_TOTAL, SEED)
    gen = egs.Problem(N_TOTAL, DTS)
    gen.set_locations(x, y)
    z = gen.generate_observations(THETA, SEED)
    gen.close()
    perm = np.random.default_rng(SEED).permutation(N_TOTAL)
    train = np.sort(perm[N_MISS:])
    return x[train].copy(), y[train].copy(), z[train].copy()


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
        "sample": f"one full evaluation at N={ns} (first {ns} training points, theta={THETA}); "
                  f"generation and solve scaled by (N/{ns})^2, potrf by (N/{ns})^3 to N={n_target}"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    import numpy as np
    from oracle import cpu_baseline as C
    from oracle import oracle as O
    # Same inputs as the B200 arm, produced on the host by the oracle's generator.
    # Z for the sampled subset only (a 41,000-point CPU Cholesky would dominate).
    t0 = time.perf_counter()
    x, y = O.generate_locations(N_TOTAL, O.GlibcRand(SEED))
    perm = np.random.default_rng(SEED).permutation(N_TOTAL)
    train = np.sort(perm[N_MISS:])
    x, y = x[train], y[train]
    n_target = len(x)
    ns = 6000
    z = O.dlarnv_normal(SEED, ns)  # any standard-normal observations: cost does not depend on Z
    _, st = C.timed_eval(x[:ns], y[:ns], z, THETA)
    per_step = 4.0
    grow = (per_step / max(sum(st.values()), 1e-3)) ** (1.0 / 3.0)
    ns = int(min(16000, max(4000, ns * grow)) // 64 * 64)
    z = O.dlarnv_normal(SEED, ns)
    a = np.zeros((ns, ns), order="F")
    for _ in range(args.warmup):
        C.timed_eval(x[:ns], y[:ns], z, THETA, a)
    scaled = []
    lat = []
    for _ in range(args.steps):
        _, st = C.timed_eval(x[:ns], y[:ns], z, THETA, a)
        scaled.append(1.0 / C.scaled_evals_per_s(st, ns, n_target))
        lat.append(sum(st.values()))
    total = sum(scaled)
    value = args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference generator semantics)",
        "config": CONFIG,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": C.threads(), "kind": "port",
                         "sample": f"each step one full evaluation at N={ns} on all host threads "
                                   f"(Matern in C/pthreads, LAPACK dpotrf/dtrtrs via OpenBLAS), scaled to "
                                   f"N={n_target} by n^2 (generation, solve) and n^3 (potrf)"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "sample_step_s_p50": statistics.median(lat), "wall_s": time.perf_counter() - t0,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-eval", action="store_true",
                    help="one evaluation between cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--profile-n", type=int, default=0,
                    help="with --profile-eval: evaluate this many of the workload's locations with "
                         "DLARNV observations instead of the full workload (small ncu captures)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)

    import numpy as np
    import torch
    import exageostat_b200 as egs

    rank, world, local = env_rank()
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    props = torch.cuda.get_device_properties(dev)
    bus = None
    try:
        bus = f"{props.pci_domain_id:08X}:{props.pci_bus_id:02X}:{props.pci_device_id:02X}.0"
    except AttributeError:
        pass

    if args.profile_eval:
        if args.profile_n:
            x, y = egs.generate_locations(args.profile_n, SEED)
            z = egs.dlarnv_normal(SEED, args.profile_n)
        else:
            x, y, z = workload_data(egs)
        p = egs.Problem(len(z), DTS)
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

    peak = fp64_dgemm_peak_tflops(torch)
    x, y, z = workload_data(egs)
    n = len(z)

    stream = torch.cuda.Stream()
    p = egs.Problem(n, DTS)
    p.set_stream(stream.cuda_stream)
    p.set_locations(x, y)
    p.set_observations(z)
    for _ in range(args.warmup):
        p.mle_eval(THETA)
    p.set_profiling(True)

    clocks = ClockSampler(bus)
    clocks.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    lat = []
    e0.record(stream)
    for _ in range(args.steps):
        t = time.perf_counter()
        ll, logdet, dot = p.mle_eval(THETA)
        lat.append(1e3 * (time.perf_counter() - t))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    clk = clocks.stop()
    if dist:
        tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    stage_ms, stage_flops, stage_launches = p.stage_stats()
    p.set_profiling(False)
    value = world * args.steps / (ms * 1e-3)

    # end to end through the host-buffer C ABI, pinned host inputs, copies in the timed region
    pin = [torch.from_numpy(a).pin_memory() for a in (x, y, z)]
    xh, yh, zh = (t.numpy() for t in pin)
    egs.mle_loglik_host(xh, yh, zh, THETA, DTS)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        ll_e2e = egs.mle_loglik_host(xh, yh, zh, THETA, DTS)
    e2e_s = time.perf_counter() - t0
    if dist:
        tt = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": 3 * n * 8 + 64,
           "d2h_bytes_per_step": 8 + 32, "api": "egs_mle_loglik_host (C ABI, host buffers)"}

    up = egs.STAGES.index("update")
    achieved = stage_flops[up] / (stage_ms[up] * 1e-3) / 1e12 if stage_ms[up] > 0 else None
    n_up = int(stage_launches[up])
    roof = {"bound": "tensor", "kernel": "dgemm_update_kernel (trailing syrk/gemm, FP64 DMMA)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": (achieved / peak) if achieved else None,
            "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 tensor; MEASURED_PEAKS.json has no FP64 entry)",
            "traffic": update_traffic_per_launch(n, DTS),
            "traffic_note": "DRAM bytes per launch: 19.0 B per updated C element (ncu, N=8000 trailing update) "
                            "times the mean block count of this workload's launches",
            "launches": n_up,
            "flops_per_launch": stage_flops[up] / max(n_up, 1)}
    eval_flops = n ** 3 / 3.0 + n ** 2 / 2.0 + n / 6.0 + n ** 2
    small = small_problem_rate(egs, torch)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (reference generator semantics, generated on device)",
        "config": dict(CONFIG, parallelism=f"replicas x{world}" if world > 1 else "single GPU"),
        "loglik": ll, "loglik_e2e": ll_e2e,
        "p50_ms": statistics.median(lat), "p99_ms": float(np.percentile(lat, 99)),
        "eval_tflops": eval_flops * world * args.steps / (ms * 1e-3) / 1e12,
        "stages_ms_per_eval": {s: float(stage_ms[i]) / args.steps for i, s in enumerate(egs.STAGES)},
        "roofline": roof, "e2e": e2e,
        "gpu_launches": int(stage_launches.sum()),
        "small_n": small,
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, info = cpu_sample(x, y, z)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": info["cores"], "kind": "port",
                                "sample": info["sample"], "stage_s": info["stage_s"]}
    p.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
