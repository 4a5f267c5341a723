"""Benchmark: D3Q19 FP32 IB-LBM sphere flow, one level step per step.

Workload (the D3Q19 FP32 configuration the headline metric is quoted on):
sphere of diameter 32 cells centred at (64,64,64) in a 256 x 128 x 128 level,
inflow U = 0.04 (ext_dir) at x-lo, foextrap at x-hi, periodic in y and z,
Re = 100, marker direct-forcing IBM with implicit velocity correction (golden
spiral markers), FP32 shifted-population storage.  A step is one
AdvancePhiAtLevel of that level: IB update_forcing + fused collide-stream.

value  : MLUPS with the state resident in HBM, device time (CUDA events on the
         library stream), max over ranks; N > 1 runs independent replicas.
e2e    : the same through the public API with the per-step host inputs copied
         in (level parameters) and the per-step result read back (the
         drag/lift force record, as the reference writes force.dat every step).
roofline: dominant kernel (fused collide-stream), algorithmic bytes 2*Q*4 per
         cell update, against the measured HBM copy bandwidth.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = dict(nx=256, ny=128, nz=128, D=32.0, center=(64.0, 64.0, 64.0), U=0.04, Re=100.0)


def set_workload_size(nx: int, ny: int, nz: int):
    """Shrinks the sphere workload (tests of the multi-rank logic on CPU);
    the sphere keeps D = ny / 4 at (nx / 4, ny / 2, nz / 2)."""
    WORKLOAD.update(nx=nx, ny=ny, nz=nz, D=ny / 4.0, center=(nx / 4.0, ny / 2.0, nz / 2.0))
METRIC = "MLUPS & % HBM roofline (D3Q19 FP32); batched/served MLUPS, p99 vs plain"
UNIT = "MLUPS"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if os.environ.get("ILBM_BENCH_BACKEND", "nccl") == "nccl" else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def allreduce_max(x: float, world: int, device) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_mlups(cells_per_rank: int, steps: int, local_ms: float, world: int, device) -> tuple:
    """Whole-job MLUPS of `world` replicas from each rank's device time: the
    cells of all ranks over the slowest rank's time (max over ranks)."""
    t_max = allreduce_max(local_ms, world, device)
    return world * cells_per_rank * steps / (t_max * 1e-3) / 1e6, t_max


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def cpu_reference_steps(steps: int, warmup: int, threads: int | None = None):
    """Times the reference's own CPU path (oracle/_ref, FP32 3D build) on the
    same workload; returns (MLUPS, seconds per step, threads, sample text)."""
    from ilbmrex_b200 import cases
    from oracle import checker
    from oracle.checker import CpuLevel
    w = WORKLOAD
    case, ib, init = cases.sphere(w["nx"], w["ny"], w["nz"], D=w["D"], center=w["center"],
                                  U=w["U"], Re=w["Re"])
    kind = "reference" if checker.available("ref", 3, fp32=True) else "port"
    threads = threads or os.cpu_count() or 1
    if kind == "reference":
        L = CpuLevel(case, "ref", fp32=True, threads=threads)
    else:
        L = CpuLevel(case, "oracle")
        threads = 1
    L.set_macro(*init())
    L.init_equilibrium()
    L.ib_create(ib)
    L.step(max(1, warmup))  # includes the one-time dense LU of the IVC operator
    t0 = time.perf_counter()
    L.step(steps)
    dt = (time.perf_counter() - t0) / steps
    sample = (f"{steps} full level steps of the {w['nx']}x{w['ny']}x{w['nz']} D3Q19 sphere "
              f"(after {max(1, warmup)} warm-up steps incl. the one-time IVC LU); "
              + ("reference sources (Source/LBM, Source/BC, Source/IBM) compiled in place, "
                 "float, restated AdvancePhiAtLevel pass structure, OpenMP"
                 if kind == "reference" else "plain-C oracle port, FP64, 1 thread"))
    return case.cells / dt / 1e6, dt, threads, kind, sample


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    steps = max(1, min(args.steps, 3))
    mlups, dt, threads, kind, sample = cpu_reference_steps(steps, 1)
    line = {"metric": METRIC, "value": round(mlups, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": steps, "warmup": 1, "ms_per_step": round(dt * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": workload_config(args),
            "cpu_baseline": {"value": round(mlups, 3), "unit": UNIT, "cores": threads,
                             "kind": kind, "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(args):
    w = WORKLOAD
    return {"workload": f"D3Q19 IB-LBM sphere, single level {w['nx']}x{w['ny']}x{w['nz']}, "
                        f"D={w['D']:g}, U={w['U']}, Re={w['Re']:g}, IVC marker IB, FP32 shifted storage",
            "lattice": "D3Q19", "cells": w["nx"] * w["ny"] * w["nz"], "storage": args.storage,
            "levels": 1, "parallelism": f"replicas{args.gpus}",
            "ib_overlap": not getattr(args, "serial", False),
            "l2_policy": "working set 637 MB > 126 MB L2 (no flush needed)"}


def run_batched(args, world, device):
    """Batched D2Q9 FP32 workload (64 seeded cylinder / pitching-airfoil cases)
    through the batch engine, against the same cases run one after another
    through the plain single-case call (ilbm_advance_level)."""
    import torch
    from ilbmrex_b200 import cases
    from ilbmrex_b200.batch import Batch
    from ilbmrex_b200.lattice import D2Q9
    from ilbmrex_b200.level import LevelSolver
    mix = cases.batch_mix(args.batch_cases)
    cells = sum(c.cells for c, _, _ in mix)
    K = args.batch_steps
    B = Batch(D2Q9, "f32", device=device.index or 0, rec_slots=512)
    for c, ib, init in mix:
        B.add(B.solver(c, ib, init), max_steps=K + 200)
    tile_w, cps, _ = B.tune(trial_steps=4)
    B.step(4)
    B.ctx.sync()
    barrier(world)
    launches0 = B.ctx.launches()
    B.ctx.record(4)
    B.step(K)
    B.ctx.record(5)
    B.ctx.sync()
    launches = B.ctx.launches() - launches0
    t_b = allreduce_max(B.ctx.elapsed_ms(4, 5), world, device)
    batched = world * cells * K / (t_b * 1e-3) / 1e6
    B.close()
    # plain: case by case through the single-case call
    Kp = args.batch_plain_steps
    t_plain = 0.0
    for c, ib, init in (mix if Kp > 0 else []):
        S = LevelSolver(c, "f32", ib=ib, device=device.index or 0)
        S.set_macro(*init())
        S.step(3)
        S.ctx.sync()
        S.ctx.record(6)
        S.step(Kp)
        S.ctx.record(7)
        S.ctx.sync()
        t_plain += S.ctx.elapsed_ms(6, 7) / Kp
        S.close()
        torch.cuda.empty_cache()
    t_plain = allreduce_max(t_plain, world, device)
    plain = world * cells / (t_plain * 1e-3) / 1e6 if Kp > 0 else None
    return {"metric": "batched MLUPS (64 D2Q9 FP32 IB cases)", "value": round(batched, 2),
            "unit": "MLUPS", "plain_case_by_case": round(plain, 2) if plain else None,
            "speedup_vs_plain": round(batched / plain, 2) if plain else None,
            "cases": len(mix), "cells": cells,
            "steps": K, "plain_steps_per_case": Kp, "ms_per_step": round(t_b / K, 4),
            "tile_w": tile_w, "ctas_per_sm": cps, "gpu_launches": int(launches),
            "workload": "seeded mix: grids 256x128..1024x512, cylinders D 16-48 Re 20-200, "
                        "NACA0012 pitching (chord 64-128, 2-15 deg, k 0.05-0.3), FP32 storage; "
                        "each case steps through its own IB (stored IVC inverse or CG)"}


def run_served(args, world, device):
    """Served mixed workload: Poisson arrivals (seeded) of D2Q9 cylinder /
    airfoil, D3Q19 duct and D3Q19 sphere requests through the continuous-
    batching server, against the same requests served one at a time through
    the plain single-case call (FIFO, same arrivals)."""
    from ilbmrex_b200.serve import Server, make_request, poisson_arrivals, run_alone
    rng = np.random.default_rng(20261203)
    n = args.serve_requests
    kinds = rng.choice(["cylinder", "duct", "sphere"], p=[0.5, 0.25, 0.25], size=n)
    reqs = [make_request(i, str(k), rng, int(rng.integers(args.serve_min_steps, args.serve_max_steps + 1)),
                         scale=args.serve_scale) for i, k in enumerate(kinds)]
    arr = poisson_arrivals(n, args.serve_rate, rng)
    for r, t in zip(reqs, arr):
        r.arrival = float(t)
    lups = sum(r.case.cells * r.steps for r in reqs)
    srv = Server("f32", device=device.index or 0, chunk=args.serve_chunk)
    stats = srv.run(reqs)
    srv.close()
    # plain: one request at a time through the single-case call
    service = []
    for r in reqs:
        t0 = time.perf_counter()
        run_alone(r, "f32", device=device.index or 0)
        service.append(time.perf_counter() - t0)
    done, lat = 0.0, []
    for r, sv in zip(reqs, service):
        done = max(done, r.arrival) + sv
        lat.append(done - r.arrival)
    plain_mlups = lups / done / 1e6  # same arrivals, one request at a time (FIFO)
    sizes = [r.case.cells for r in reqs]
    return {"metric": "served MLUPS, mixed D2Q9/D3Q19 FP32 requests", "value": round(stats["mlups"], 2),
            "unit": "MLUPS", "p50_latency_s": round(stats["p50_latency_s"], 4),
            "p99_latency_s": round(stats["p99_latency_s"], 4),
            "plain_mlups": round(plain_mlups, 2),
            "plain_p50_latency_s": round(float(np.percentile(lat, 50)), 4),
            "plain_p99_latency_s": round(float(np.percentile(lat, 99)), 4),
            "speedup_vs_plain": round(stats["mlups"] / plain_mlups, 2),
            "requests": n, "arrival_rate_per_s": args.serve_rate, "makespan_s": round(stats["makespan_s"], 3),
            "plain_makespan_s": round(done, 3), "plain_busy_s": round(sum(service), 3),
            "server_time_s": stats["time_s"],
            "cells_min_max": [int(min(sizes)), int(max(sizes))],
            "steps_min_max": [args.serve_min_steps, args.serve_max_steps],
            "workload": f"seeded Poisson arrivals; 50% D2Q9 cylinder/airfoil, 25% D3Q19 duct N x N x 4N, "
                        f"25% D3Q19 sphere; grid edges scaled by {args.serve_scale} and step counts "
                        f"{args.serve_min_steps}-{args.serve_max_steps} (the served configuration's "
                        f"1e5-3e7 cells x 1000-20000 steps shrunk to a bench-sized run)"}


def run_b200(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    from ilbmrex_b200 import capi, cases
    from ilbmrex_b200.level import LevelSolver

    if args.only_batched or args.only_served:  # profiling aids: one workload alone
        out = run_batched(args, world, device) if args.only_batched else run_served(args, world, device)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return

    w = WORKLOAD
    case, ib, init = cases.sphere(w["nx"], w["ny"], w["nz"], D=w["D"], center=w["center"],
                                  U=w["U"], Re=w["Re"])
    S = LevelSolver(case, args.storage, ib=ib, device=local)
    S.set_macro(*init())
    ctx = S.ctx
    cells = case.cells
    q = case.lattice.q
    sbytes = {"f64": 8, "f32": 4, "f16": 2}[args.storage]
    B_cell = 2 * q * sbytes

    # ---- device-resident timed region -----------------------------------
    K = args.steps

    def one_step(s_idx=None, serial=False):
        use_macro = S.macro if S.first_step_macro else None
        b = S._box(S.f, S.f_next, macro_in=use_macro, force=S.force_cur, force_prev=S.force_prev)
        if serial:
            capi.check(S.L.ilbm_ib_update_forcing(S.ib, C.byref(b), C.byref(S.params), case.dt,
                                                  S.time), "ib")
            if s_idx is not None:
                ctx.record(16 + 2 * s_idx)
            capi.check(S.L.ilbm_level_step(ctx.h, C.byref(b), 1, C.byref(S.params)), "step")
            if s_idx is not None:
                ctx.record(17 + 2 * s_idx)
        else:
            capi.check(S.L.ilbm_advance_level(ctx.h, C.byref(b), C.byref(S.params), S.ib,
                                              case.dt, S.time), "advance_level")
        S.f, S.f_next = S.f_next, S.f
        S.force_cur, S.force_prev = S.force_prev, S.force_cur
        S.first_step_macro = False
        S.time += case.dt
        S.istep += 1

    # first step: includes the one-time IVC operator set-up (stored inverse)
    ctx.sync()
    ctx.record(2)
    one_step(serial=args.serial)
    ctx.record(3)
    ctx.sync()
    first_step_ms = ctx.elapsed_ms(2, 3)
    for _ in range(max(3, args.warmup) - 1):
        one_step(serial=args.serial)
    ctx.sync()
    torch.cuda.synchronize(device)

    launches0 = ctx.launches()
    sampler = ClockSampler(local)
    with sampler:
        barrier(world)
        ctx.sync()
        ctx.record(0)
        for s in range(K):
            one_step(serial=args.serial)
        ctx.record(1)
        ctx.sync()
        barrier(world)
    launches = ctx.launches() - launches0
    t_ms = ctx.elapsed_ms(0, 1)
    value, t_max = aggregate_mlups(cells, K, t_ms, world, device)
    clocks = sampler.summary()

    # ---- roofline pass: the level step (ghost-shell push + fused collide-
    # stream) bracketed by events, IB chain outside the brackets ------------
    Kr = max(3, min(K, 20))
    for s in range(Kr):
        one_step(s, serial=True)
    ctx.sync()
    step_ms = [ctx.elapsed_ms(16 + 2 * s, 17 + 2 * s) for s in range(Kr)]
    kern_ms = float(np.mean(step_ms))
    peak, peak_kind = peaks()
    achieved = B_cell * cells / (kern_ms * 1e-3) / 1e9

    # ---- end-to-end through the public API --------------------------------
    Ke = max(3, min(K, 20))
    ctx.sync()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(Ke):
        S.advance_phi_at_level(record_force=True)  # reads Cd/Cl back every step
    ctx.sync()
    e2e_s = allreduce_max(time.perf_counter() - t0, world, device)
    e2e = world * cells * Ke / e2e_s / 1e6
    h2d = C.sizeof(capi.LevelParams_t) + C.sizeof(capi.Box_t) + 16
    d2h = 3 * 8 + 3 * 8 + 4

    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get("k_step_d3q19_f32_bytes_per_launch")
        except Exception:
            traffic = None

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            mlups, dt, threads, kind, sample = cpu_reference_steps(2, 1)
            cpu_base = {"value": round(mlups, 3), "unit": UNIT, "cores": threads, "kind": kind,
                        "sample": sample}
        except Exception as e:  # the checker is optional at run time
            cpu_base = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                        "sample": f"unavailable: {e}"}

    batched = None
    if not args.no_batched:
        batched = run_batched(args, world, device)
    served = None
    if not args.no_served:
        served = run_served(args, world, device)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": max(3, args.warmup), "ms_per_step": round(t_max / K, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage != "f64" else "f64", "data": "synthetic",
            "config": workload_config(args),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": "level step = k_step<D3Q19,F32_SHIFT> (ghost-shell push in its leading blocks)",
                         "kernel_ms": round(kern_ms, 4), "bytes_per_cell": B_cell,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6650 GB/s"},
            "cpu_baseline": cpu_base,
            "e2e": {"value": round(e2e, 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "ib_markers": S.num_markers(),
            "ivc_cg_iterations": S.cg_iterations(),
            "first_step_ms_incl_ivc_setup": round(first_step_ms, 2),
            "batched": batched,
            "served": served,
        }
        print(json.dumps(line), flush=True)
    S.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f64", "f32", "f16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=0, help="sphere level size override (tests)")
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--nz", type=int, default=0)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched workload")
    ap.add_argument("--no-served", action="store_true", help="skip the served workload")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-rate", type=float, default=200.0, help="arrivals per second")
    ap.add_argument("--serve-scale", type=float, default=0.5)
    ap.add_argument("--serve-min-steps", type=int, default=300)
    ap.add_argument("--serve-max-steps", type=int, default=1500)
    ap.add_argument("--serve-chunk", type=int, default=100)
    ap.add_argument("--only-batched", action="store_true",
                    help="run only the batched workload and print its result (profiling aid)")
    ap.add_argument("--only-served", action="store_true",
                    help="run only the served workload and print its result (profiling aid)")
    ap.add_argument("--batch-cases", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=40)
    ap.add_argument("--batch-plain-steps", type=int, default=8)
    ap.add_argument("--serial", action="store_true",
                    help="run the IB chain and the level step one after the other (no overlap)")
    args = ap.parse_args()
    if args.nx:
        set_workload_size(args.nx, args.ny or args.nx // 2, args.nz or args.nx // 2)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
