"""Throughput of LB3D's per-timestep hot path on B200.

Default workload (one GPU): the ternary amphiphilic D3Q19 system of
128^3 sites, periodic, FP32-deviation storage (red, blue and surfactant at
rho 0.7 + U(-0.01, 0.01), random unit dipoles, g_br = 0.08, g_bs = -0.006,
g_ss = -0.0045, tau = tau_d = 1, beta = 10), the configuration the headline
MLUPS is quoted on.  A "step" is one full time step (stages 6..9 of
lb3d_time_loop) over the whole lattice.  The FP64 drop-in path is measured
on the same system and reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one independent lattice per rank (replicas: the path has no data
exchange between lattices), timed on the device as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ternary D3Q19 MLUPS & %HBM peak, FP32-dev vs FP64; ensemble solves/s, p99 lat"
L = 128
BYTES_PER_SITE = {("f32", 3): 480, ("f32", 2): 304, ("f64", 3): 960, ("f64", 2): 608}
PHYS = dict(tau_d=1.0, g_br=0.08, g_bs=-0.006, g_ss=-0.0045, beta=10.0, d_0=1.0, bdist=2, restore=1)


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def workload_params(L=L, ncomp=3, precision=1):
    from lb3d_b200.config import Params
    return Params(nx=L, ny=L, nz=L, ncomp=ncomp, precision=precision, **PHYS).finalize()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(threads, seconds_target=15.0):
    """The CPU restatement (oracle port) of the same workload on the host cores:
    the reference's own Fortran/MPI build needs gfortran and MPI, which this
    image does not have."""
    from lb3d_b200.ic import uniform_mixture
    from tests._oracle import Oracle
    p = workload_params(precision=0)
    o = Oracle(p, uniform_mixture(L, L, L, 3, seed=1), threads=threads)
    o.run(1)  # warm-up
    steps, t0 = 0, time.perf_counter()
    while True:
        o.run(1)
        steps += 1
        if time.perf_counter() - t0 > seconds_target or steps >= 20:
            break
    dt = time.perf_counter() - t0
    return {"value": round(L ** 3 * steps / dt / 1e6, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
            "sample": f"ternary {L}^3 FP64 CPU restatement, {steps} full steps ({dt:.1f} s), OpenMP"}


def run_reference(args):
    """--impl reference: the CPU restatement of the reference's path on all
    host threads, same workload and metric; rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from lb3d_b200.ic import uniform_mixture
    from tests._oracle import Oracle
    threads = os.cpu_count() or 1
    p = workload_params(precision=0)
    o = Oracle(p, uniform_mixture(L, L, L, 3, seed=1), threads=threads)
    o.run(max(1, min(args.warmup, 3)))
    steps = max(1, min(args.steps, 10))
    t0 = time.perf_counter()
    o.run(steps)
    dt = time.perf_counter() - t0
    v = L ** 3 * steps / dt / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 3), "unit": "MLUPS",
        "n_gpus": args.gpus, "steps": steps, "warmup": args.warmup, "ms_per_step": round(1e3 * dt / steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"ternary D3Q19 {L}^3 periodic (FP64, CPU)", "lattice": [L, L, L]},
        "cpu_baseline": {"value": round(v, 3), "unit": "MLUPS", "cores": threads, "kind": "port",
                         "sample": f"full {L}^3 lattice, {steps} steps; the reference's Fortran/MPI build is "
                                   "unavailable in this image (no gfortran, no MPI), so its C++ restatement runs"},
        "e2e": {"value": round(v, 3), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def time_lattice(lat, steps, warmup, stream_ptr):
    import torch
    st = torch.cuda.ExternalStream(stream_ptr)
    lat.time_loop(warmup)
    lat.sync()
    lat.set_profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    lat.time_loop(steps)
    e1.record(st)
    e1.synchronize()
    wall_ms = e0.elapsed_time(e1)
    kms, klaunch, alllaunch = lat.kernel_stats()
    lat.set_profiling(False)
    return wall_ms, kms, klaunch, alllaunch


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from lb3d_b200.ic import uniform_mixture
    from lb3d_b200.lib import Lattice

    peak, peak_kind = measured_peak()
    state = uniform_mixture(L, L, L, 3, seed=1 + rank)
    N = L ** 3

    # ---- FP32 deviation path (headline) ----
    lat = Lattice(workload_params(precision=1))
    lat.upload_state(state)
    shape, tune_ms = lat.autotune()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall_ms, kms, klaunch, alllaunch = time_lattice(lat, args.steps, args.warmup, lat.stream)
    t = torch.tensor([wall_ms, kms], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.barrier()
    wall_ms, kms = float(t[0]), float(t[1])
    ms_step = wall_ms / args.steps
    value = world * N * args.steps / (wall_ms * 1e-3) / 1e6
    per_launch_ms = kms / max(klaunch, 1)
    alg_bytes = BYTES_PER_SITE[("f32", 3)] * N
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    lat.close()

    # ---- FP64 drop-in path on the same system ----
    lat64 = Lattice(workload_params(precision=0))
    lat64.upload_state(state)
    s64 = max(5, args.steps // 5)
    w64, k64, n64, _ = time_lattice(lat64, s64, 3, lat64.stream)
    t64 = torch.tensor([w64], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(t64, op=dist.ReduceOp.MAX)
    w64 = float(t64[0])
    v64 = world * N * s64 / (w64 * 1e-3) / 1e6
    lat64.close()

    # ---- end to end through the C-ABI with host buffers ----
    # one solve = upload of the FP64 restart state from pinned host memory,
    # `steps` time steps, download of the populations to host memory
    host = {k: (torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy() if v is not None else None)
            for k, v in state.items() if k in ("n", "db", "rock")}
    lat = Lattice(workload_params(precision=1))
    lat.set_launch_shape(*shape)
    out_n = torch.empty(tuple(state["n"].shape), dtype=torch.float64).pin_memory().numpy()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    lat.upload(host["n"], host["db"], host["rock"])
    lat.time_loop(args.steps)
    from lb3d_b200.lib import lib, ptr
    lib().lb3dc_download_state(lat.h, ptr(out_n), None, None, None, None)
    e2e_s = time.perf_counter() - t0
    te = torch.tensor([e2e_s], device="cuda", dtype=torch.float64)
    if world > 1:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_s = float(te[0])
    lat.close()
    h2d = sum(v.nbytes for v in host.values() if v is not None)
    d2h = out_n.nbytes

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(os.cpu_count() or 1)
        except Exception as exc:  # report, do not fail the bench
            cpu = {"value": None, "error": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded rho = 0.7 + U(-0.01,0.01) per component, unit dipoles",
            "config": {"workload": f"ternary D3Q19 {L}^3 periodic, FP32-deviation storage, fused stream-collide",
                       "lattice": [L, L, L], "g_br": 0.08, "g_bs": -0.006, "g_ss": -0.0045, "tau": 1.0,
                       "tau_d": 1.0, "beta": 10.0, "parallelism": f"replicas x{world}",
                       "l2": f"populations {2 * 57 * 4 * N / 1e6:.0f} MB > 126 MB L2, no flush",
                       "launch_shape": list(shape)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": None, "peak_kind": peak_kind,
                         "bytes_per_site": BYTES_PER_SITE[("f32", 3)], "kernel_ms": round(per_launch_ms, 4)},
            "fp64_plain": {"value": round(v64, 1), "unit": "MLUPS", "steps": s64,
                           "achieved_gbs": round(BYTES_PER_SITE[("f64", 3)] * N / (w64 / s64 * 1e-3) / 1e9, 1),
                           "frac": round(BYTES_PER_SITE[("f64", 3)] * N / (w64 / s64 * 1e-3) / 1e9 / peak, 4),
                           "fp32_over_fp64": round(value / v64, 3)},
            "e2e": {"value": round(world * N * args.steps / e2e_s / 1e6, 1), "unit": "MLUPS",
                    "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                    "solve": f"upload FP64 state + {args.steps} steps + download populations"},
            "gpu_launches": int(alllaunch),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
