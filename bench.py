"""Throughput of LB3D's per-timestep hot path on B200.

Default workload (one GPU): the ternary amphiphilic D3Q19 system of
128^3 sites, periodic, FP32-deviation storage (red, blue and surfactant at
rho 0.7 + U(-0.01, 0.01), random unit dipoles, g_br = 0.08, g_bs = -0.006,
g_ss = -0.0045, tau = tau_d = 1, beta = 10), the configuration the headline
MLUPS is quoted on.  A "step" is one full time step (stages 6..9 of
lb3d_time_loop) over the whole lattice.  Beside it the line reports the FP64
drop-in path on the same system, the serving ensemble (Poisson stream of
ternary parameter-sweep solves, continuous batching) against sequential
plain-path solves, and the CPU restatement on the host cores.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

N > 1 runs one independent lattice per rank and splits the request stream
over the ranks (replicas: the path has no data exchange between lattices);
device times are maxima over ranks.
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
# DRAM bytes per site and step that ncu measured (dram__bytes_read.sum +
# dram__bytes_write.sum of the moments, dipole and staged collide passes) on
# the ternary 128^3 workload, keyed by (tile x, tile y, strategy); captured
# with 8-plane chunks (the chunk depth moves only the ring halo reloads,
# under 1 % of this figure).
NCU_TRAFFIC_PER_SITE = {(32, 4, 2): 772}
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

    FIELDS = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []
        self.recording = False

    def __enter__(self):
        q = "clocks.sm,clocks.max.sm,power.draw," + ",".join("clocks_event_reasons." + f for f in self.FIELDS)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            time.sleep(0.5)  # let the sampler start
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            if self.recording:
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
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(self.FIELDS, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_baseline(threads, seconds_target=15.0):
    """The CPU restatement (oracle port) of the same workload on the host
    cores: the reference's own Fortran/MPI build needs gfortran and MPI,
    which this image does not have."""
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
    from lb3d_b200.dist import world
    rank, _, size = world()
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


def time_lattice(lat, steps, warmup, sampler=None):
    import torch
    st = torch.cuda.ExternalStream(lat.stream)
    lat.time_loop(warmup)
    lat.sync()
    lat.set_profiling(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if sampler:
        sampler.recording = True
    e0.record(st)
    lat.time_loop(steps)
    e1.record(st)
    e1.synchronize()
    if sampler:
        sampler.recording = False
    wall_ms = e0.elapsed_time(e1)
    kms, klaunch, alllaunch = lat.kernel_stats()
    lat.set_profiling(False)
    return wall_ms, kms, klaunch, alllaunch


def serving(rank, size, nreq=96, seq_sample=4):
    """The serving ensemble on this rank's share of a seeded Poisson stream
    of ternary parameter-sweep solves (mean 200 req/s, cubic edges
    log-uniform 16..96, steps 500..5000), continuous batching by HBM
    footprint; and sequential solves of the first requests through the FP64
    plain path and the single-lattice FP32 path for comparison."""
    from lb3d_b200.dist import partition
    from lb3d_b200.ensemble import Ensemble, Server, sweep_requests
    from lb3d_b200.ic import uniform_mixture
    from lb3d_b200.lib import Lattice
    reqs = partition(sweep_requests(nreq, seed=7), rank, size)
    ens = Ensemble(3, capacity_sites=24_000_000, max_lattices=2048, shape=(32, 4, 8, 2))
    out = Server(ens, chunk=512, download=True, on_result=lambda r, res: None).run(reqs)
    ens.close()
    seq = {}
    sample = reqs[:seq_sample]
    for prec, name in ((0, "fp64_plain"), (1, "fp32_single")):
        t = 0.0
        for r in sample:
            p = r.params
            st = uniform_mixture(p.nx, p.ny, p.nz, 3, seed=r.seed)
            lat = Lattice(p, precision=prec)
            t0 = time.perf_counter()
            lat.upload_state(st)
            lat.time_loop(r.steps)
            lat.download()
            t += time.perf_counter() - t0
            lat.close()
        seq[name] = len(sample) / t
    return out, seq, len(sample)


def run_configs(args):
    """--configs: the four single-lattice workloads on one GPU, one JSON line each (MLUPS,
    fraction of the HBM roofline, and for ternary 128^3 the FP32-vs-FP64 error
    after 1k and 10k steps)."""
    import torch
    from lb3d_b200.config import Params
    from lb3d_b200.ic import invasion_state, sphere_pack, uniform_mixture
    from lb3d_b200.lib import Lattice
    torch.cuda.set_device(0)
    peak, _ = measured_peak()

    def mlups(p, st, prec, steps, tune=False):
        lat = Lattice(p, precision=prec)
        lat.upload_state(st)
        shape = None
        if prec == 1 and tune:
            shape, _ = lat.autotune()
        w, k, n, _ = time_lattice(lat, steps, 5)
        lat.close()
        return p.nx * p.ny * p.nz * steps / (w * 1e-3) / 1e6, shape

    def line(d):
        print(json.dumps(d), flush=True)

    phys2 = dict(tau_d=1.0, beta=10.0, d_0=1.0, bdist=2, restore=1, g_br=0.08)
    # binary 64^3 FP64, 1000 steps
    p1 = Params(nx=64, ny=64, nz=64, ncomp=2, **phys2).finalize()
    st1 = uniform_mixture(64, 64, 64, 2, seed=1)
    v, _ = mlups(p1, st1, 0, 1000)
    line({"case": "binary-64", "workload": "binary 64^3 periodic FP64 plain, 1000 steps", "mlups": round(v, 1),
          "frac": round(v * 1e6 * 608 / 1e9 / peak, 4), "bytes_per_site": 608})
    # ternary 128^3, FP64 vs FP32 deviation error after 1k and 10k steps
    p2 = workload_params(precision=0)
    st2 = uniform_mixture(L, L, L, 3, seed=1)
    a = Lattice(p2, precision=0)
    b = Lattice(p2, precision=1)
    a.upload_state(st2)
    b.upload_state(st2)
    b.autotune()
    done = 0
    for target in (1000, args.error_steps):
        a.time_loop(target - done)
        b.time_loop(target - done)
        done = target
        ra, rb = a.download(), b.download()
        d = np.abs(ra["rho"] - rb["rho"])
        phi_a, phi_b = ra["rho"][0] - ra["rho"][1], rb["rho"][0] - rb["rho"][1]
        line({"case": "ternary-128-error", "steps": target, "workload": "ternary 128^3, FP32-deviation vs FP64 plain",
              "max_abs_drho": float(d.max()), "rms_drho": float(np.sqrt((d ** 2).mean())),
              "max_abs_dphi": float(np.abs(phi_a - phi_b).max()),
              "rho_range_fp64": [float(ra["rho"].min()), float(ra["rho"].max())],
              "max_abs_ddb": float(np.abs(ra["db"] - rb["db"]).max())})
    a.close()
    b.close()
    # binary Lees-Edwards 256x128x128 (x-planes sheared), shear 0.05
    p3 = Params(nx=256, ny=128, nz=128, ncomp=2, boundary_cond=-1, inv_fluid=5, shear_u=0.05,
                **phys2).finalize()
    st3 = uniform_mixture(256, 128, 128, 2, seed=3)
    v32, shape3 = mlups(p3, st3, 1, 200, tune=True)
    v64, _ = mlups(p3, st3, 0, 200)
    line({"case": "lees-edwards-256x128x128",
          "workload": "binary Lees-Edwards 256x128x128 (x-planes sheared, shear_u 0.05), FP32 deviation "
                      "with FP64 plane offset, and FP64 plain",
          "mlups_fp32": round(v32, 1), "frac_fp32": round(v32 * 1e6 * 304 / 1e9 / peak, 4),
          "mlups_fp64": round(v64, 1), "frac_fp64": round(v64 * 1e6 * 608 / 1e9 / peak, 4),
          "launch_shape": shape3})
    # binary porous 256^3, body force 1e-5 along x, red inlet slab
    rock = sphere_pack(256, 256, 256, seed=4, porosity=0.4, rmin=6, rmax=12, overlap=True)
    por = 1.0 - float(rock.mean())
    p4 = Params(nx=256, ny=256, nz=256, ncomp=2, g_accn_x=1e-5, **phys2).finalize()
    st4 = invasion_state(256, 256, 256, rock, seed=4)
    v32, shape = mlups(p4, st4, 1, 200, tune=True)
    v64, _ = mlups(p4, st4, 0, 50)
    nf = por
    line({"case": "porous-256", "workload": "binary porous 256^3 (overlapping spheres r 6..12), body force 1e-5",
          "porosity": round(por, 4), "mlups_fp32": round(v32, 1), "mlups_fp64": round(v64, 1),
          "frac_fp32": round(v32 * 1e6 * (304 * nf + 1) / 1e9 / peak, 4), "launch_shape": shape})


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--requests", type=int, default=96)
    ap.add_argument("--configs", action="store_true", help="measure the four single-lattice workloads (binary 64^3 FP64, ternary 128^3 FP32 error, "
                    "Lees-Edwards 256x128x128, porous 256^3) instead")
    ap.add_argument("--error-steps", type=int, default=10000)
    ap.add_argument("--shape", default=None,
                    help="tx,ty,zc,split: fixed FP32 launch shape instead of the autotuner (profiling runs)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.configs:
        return run_configs(args)

    import torch
    from lb3d_b200 import dist as D
    rank, local, world = D.world()
    torch.cuda.set_device(local)
    pg = D.init("nccl")
    from lb3d_b200.ic import uniform_mixture
    from lb3d_b200.lib import Lattice, lib, ptr

    peak, peak_kind = measured_peak()
    state = uniform_mixture(L, L, L, 3, seed=D.replica_seed(1, rank))
    N = L ** 3
    dev = "cuda"

    # ---- FP32 deviation path (headline) ----
    lat = Lattice(workload_params(precision=1))
    lat.upload_state(state)
    if args.shape:
        lat.set_launch_shape(*[int(v) for v in args.shape.split(",")])
        shape = lat.launch_shape
    else:
        shape, tune_ms = lat.autotune()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        wall_ms, kms, klaunch, alllaunch = time_lattice(lat, args.steps, args.warmup, clk)
    wall_ms, kms = D.max_over_ranks([wall_ms, kms], dev)
    ms_step = wall_ms / args.steps
    value = world * N * args.steps / (wall_ms * 1e-3) / 1e6
    per_step_ms = kms / max(klaunch, 1)
    alg_bytes = BYTES_PER_SITE[("f32", 3)] * N
    achieved = alg_bytes / (per_step_ms * 1e-3) / 1e9
    lat.close()

    # ---- FP64 drop-in path on the same system ----
    lat64 = Lattice(workload_params(precision=0))
    lat64.upload_state(state)
    s64 = max(20, args.steps // 5)
    w64, k64, n64, _ = time_lattice(lat64, s64, 3)
    (w64,) = D.max_over_ranks([w64], dev)
    v64 = world * N * s64 / (w64 * 1e-3) / 1e6
    lat64.close()

    # ---- end to end through the C-ABI with host buffers ----
    # one solve = upload of the FP64 restart state from pinned host memory,
    # `steps` time steps, download of the FP64 populations to pinned memory
    host = {k: torch.from_numpy(np.ascontiguousarray(v)).pin_memory().numpy()
            for k, v in state.items() if k in ("n", "db", "rock") and v is not None}
    lat = Lattice(workload_params(precision=1))
    lat.set_launch_shape(*shape)
    out_n = torch.empty(tuple(state["n"].shape), dtype=torch.float64).pin_memory().numpy()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    t0 = time.perf_counter()
    lat.upload(host["n"], host.get("db"), host.get("rock"))
    t1 = time.perf_counter()
    lat.time_loop(args.steps)
    lat.sync()
    t2 = time.perf_counter()
    lib().lb3dc_download_state(lat.h, ptr(out_n), None, None, None, None)
    t3 = time.perf_counter()
    (e2e_s,) = D.max_over_ranks([t3 - t0], dev)
    e2e_parts = {"upload_ms": round((t1 - t0) * 1e3, 2), "steps_ms": round((t2 - t1) * 1e3, 2),
                 "download_ms": round((t3 - t2) * 1e3, 2)}
    lat.close()
    h2d = sum(v.nbytes for v in host.values())
    d2h = out_n.nbytes

    # ---- serving ensemble ----
    serve = None
    if not args.no_serving:
        out, seq, nseq = serving(rank, world, args.requests)
        wall, = D.max_over_ranks([out["wall_s"]], dev)
        solves, su = D.sum_over_ranks([out["solves"], out["site_updates"]], dev)
        p99, = D.max_over_ranks([out["p99_s"]], dev)
        serve = {"requests": args.requests, "solves_per_s": round(solves / wall, 3),
                 "p50_s": round(out["p50_s"], 3), "p99_s": round(p99, 3),
                 "glups": round(su / wall / 1e9, 3),
                 "sequential_fp64_plain_solves_per_s": round(world * seq["fp64_plain"], 3),
                 "sequential_fp32_single_solves_per_s": round(world * seq["fp32_single"], 3),
                 "speedup_vs_sequential_fp64": round(solves / wall / (world * seq["fp64_plain"]), 2),
                 "sequential_sample": nseq,
                 "stream": "Poisson 200 req/s, L log-uniform 16..96, steps 500..5000, g_br/g_bs/g_ss swept"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            cpu = cpu_baseline(os.cpu_count() or 1)
        except Exception as exc:  # reported, does not fail the bench
            cpu = {"value": None, "error": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded rho = 0.7 + U(-0.01,0.01) per component, unit dipoles",
            "config": {"workload": f"ternary D3Q19 {L}^3 periodic, FP32-deviation storage",
                       "lattice": [L, L, L], "g_br": 0.08, "g_bs": -0.006, "g_ss": -0.0045, "tau": 1.0,
                       "tau_d": 1.0, "beta": 10.0, "parallelism": f"replicas x{world}",
                       "l2": f"populations {2 * 57 * 4 * N / 1e6:.0f} MB > 126 MB L2, no flush",
                       "launch_shape": list(shape[:3]),
                       "strategy": ["fused", "split", "split, staged collide"][shape[3]],
                       "shape_source": "fixed" if args.shape else "autotuned"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4),
                         "traffic": (NCU_TRAFFIC_PER_SITE[(shape[0], shape[1], shape[3])] * N
                                     if (shape[0], shape[1], shape[3]) in NCU_TRAFFIC_PER_SITE else None),
                         "traffic_note": "DRAM bytes per step from one ncu capture of the three passes "
                                         "(null for launch shapes without a capture)",
                         "peak_kind": peak_kind,
                         "bytes_per_site": BYTES_PER_SITE[("f32", 3)], "kernel_ms_per_step": round(per_step_ms, 4)},
            "fp64_plain": {"value": round(v64, 1), "unit": "MLUPS", "steps": s64,
                           "achieved_gbs": round(BYTES_PER_SITE[("f64", 3)] * N / (w64 / s64 * 1e-3) / 1e9, 1),
                           "frac": round(BYTES_PER_SITE[("f64", 3)] * N / (w64 / s64 * 1e-3) / 1e9 / peak, 4),
                           "fp32_over_fp64": round(value / v64, 3)},
            "ensemble": serve,
            "e2e": {"value": round(world * N * args.steps / e2e_s / 1e6, 1), "unit": "MLUPS",
                    "h2d_bytes_per_step": int(h2d / args.steps), "d2h_bytes_per_step": int(d2h / args.steps),
                    "solve": f"upload FP64 state + {args.steps} steps + download FP64 populations",
                    **e2e_parts},
            "gpu_launches": int(alllaunch),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
