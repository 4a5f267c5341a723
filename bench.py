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
         drag/lift force record, as the reference writes force.dat every step;
         each step's record lands in pinned host memory and is taken by the
         host once the next step is queued), wall clock, on a fresh hierarchy
         with the same warm-up, so both legs time the same steps of the flow.
roofline: dominant kernel (fused collide-stream), algorithmic bytes 2*Q*4 per
         cell update, against the measured HBM copy bandwidth.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
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


def refined_box():
    """Base-cell box [lo, hi) of the refined level around the sphere: one
    diameter upstream and across, two downstream (32..128 x 32..96 x 32..96
    for the 256 x 128 x 128 grid), kept two base cells inside the domain."""
    w = WORKLOAD
    n = (w["nx"], w["ny"], w["nz"])
    c, D = w["center"], w["D"]
    lo = [int(math.floor(c[0] - D)), int(math.floor(c[1] - D)), int(math.floor(c[2] - D))]
    hi = [int(math.ceil(c[0] + 2 * D)), int(math.ceil(c[1] + D)), int(math.ceil(c[2] + D))]
    lo = [max(lo[a], 2) for a in range(3)]
    hi = [min(hi[a], n[a] - 2) for a in range(3)]
    return tuple(lo), tuple(hi)


def sphere_hierarchy():
    from ilbmrex_b200 import cases
    w = WORKLOAD
    lo, hi = refined_box()
    return cases.sphere_two_level(w["nx"], w["ny"], w["nz"], D=w["D"], center=w["center"], U=w["U"],
                                  Re=w["Re"], box_lo=lo, box_hi=hi)
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
            self._stop.wait(0.05)

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


def cpu_reference_levels(levels, steps: int, warmup: int, threads: int | None = None,
                         budget_s: float = 120.0):
    """Times the reference's own CPU level step (oracle/_ref: Source/LBM,
    Source/BC compiled in place, float build, the restated AdvancePhiAtLevel
    pass structure, OpenMP) on each (case, init, weight) of `levels`: per
    level `warmup` untimed steps, then up to `steps` timed ones (fewer when
    the first timed step shows that `steps` would exceed budget_s in all).
    Returns (seconds per weighted step = sum of weight x level step time,
    threads, kind, steps timed)."""
    from oracle import checker
    from oracle.checker import CpuLevel
    dim = levels[0][0].dim
    kind = "reference" if checker.available("ref", dim, fp32=True) else "port"
    threads = threads or os.cpu_count() or 1
    total, timed = 0.0, steps
    for case, init, weight in levels:
        if kind == "reference":
            L = CpuLevel(case, "ref", fp32=True, threads=threads)
        else:
            L = CpuLevel(case, "oracle")
            threads = 1
        L.set_macro(*init())
        L.init_equilibrium()
        L.step(max(1, warmup))
        t0 = time.perf_counter()
        L.step(1)
        first = time.perf_counter() - t0
        n = max(1, min(timed, int(budget_s / max(first * len(levels) * weight, 1e-9))))
        timed = min(timed, n)
        if n > 1:
            t0 = time.perf_counter()
            L.step(n - 1)
            per = (first + time.perf_counter() - t0) / n
        else:
            per = first
        total += weight * per
        L.close()
    return total, threads, kind, timed


def cpu_reference_steps(steps: int, warmup: int, threads: int | None = None):
    """The reference's CPU level step on the levels of the sphere hierarchy:
    MLUPS = updates of one coarse step (coarse + 2 x fine cells) over (coarse
    step time + 2 x fine step time).  Returns (MLUPS, seconds per coarse
    step, threads, kind, steps timed, sample text)."""
    tl, ib, ic, if_ = sphere_hierarchy()
    dt, threads, kind, timed = cpu_reference_levels(
        [(tl.coarse, ic, 1.0), (tl.fine_box(), if_, 2.0)], steps, warmup, threads)
    updates = tl.coarse.cells + 2 * int(np.prod(tl.fine_n_cell))
    sample = (f"{timed} level steps each of the coarse level ({tl.coarse.cells} cells) and of the fine box "
              f"({int(np.prod(tl.fine_n_cell))} cells) after {max(1, warmup)} warm-up step(s), timed as "
              "coarse + 2 x fine per coarse step; "
              + ("reference sources (Source/LBM, Source/BC) compiled in place, float, restated "
                 "AdvancePhiAtLevel pass structure, OpenMP" if kind == "reference"
                 else "plain-C oracle port, FP64, 1 thread"))
    return updates / dt / 1e6, dt, threads, kind, timed, sample


REFERENCE_SCOPE = ("the reference's level step (collide with Guo forcing, bounce-back, stream, "
                   "macro) on both levels of the hierarchy, float build on all host cores; NOT "
                   "included: the immersed body's update_forcing (its 12,869-marker dense LU alone runs "
                   "for minutes on the host; see with_body_single_level for its per-step cost on the "
                   "single-level sphere) and the coarse-fine fill / average-down (AMReX's)")


def cpu_reference_body(warmup: int, steps: int = 3, threads: int | None = None):
    """The reference's CPU path WITH its body on the sphere's base level
    alone (3,218 markers): IBMarkerDF::update_forcing compiled in place (its
    one-time dense LU inside the untimed warm-up) plus the level step, against
    the same level without the body."""
    from oracle import checker
    from oracle.checker import CpuLevel
    from ilbmrex_b200 import cases
    if not checker.available("ref", 3, fp32=True):
        return None
    w = WORKLOAD
    case, ib, init = cases.sphere(w["nx"], w["ny"], w["nz"], D=w["D"], center=w["center"], U=w["U"],
                                  Re=w["Re"])
    threads = threads or os.cpu_count() or 1
    out = {}
    for with_body in (False, True):
        L = CpuLevel(case, "ref", fp32=True, threads=threads)
        L.set_macro(*init())
        L.init_equilibrium()
        if with_body:
            L.ib_create(ib)
        L.step(max(1, warmup))
        t0 = time.perf_counter()
        L.step(steps)
        out[with_body] = (time.perf_counter() - t0) / steps
        if with_body:
            n_mark = L.num_markers()
        L.close()
    return {"mlups": round(case.cells / out[True] / 1e6, 3), "ms_per_step": round(out[True] * 1e3, 1),
            "ms_per_step_without_body": round(out[False] * 1e3, 1),
            "ib_ms_per_step": round((out[True] - out[False]) * 1e3, 1), "markers": int(n_mark),
            "cores": threads, "steps": steps,
            "sample": f"sphere base level {w['nx']}x{w['ny']}x{w['nz']} alone, {steps} steps with and "
                      f"without its body after {max(1, warmup)} warm-up step(s) (the IVC dense LU in the "
                      "first); reference sources incl. Source/IBM/IBMarkerDF.cpp compiled in place, float, "
                      "OpenMP"}


def run_reference(args):
    world, rank, local = dist_setup()
    if rank != 0:
        return
    warm = max(3, args.warmup)
    mlups, dt, threads, kind, timed, sample = cpu_reference_steps(max(1, args.steps), warm)
    body = cpu_reference_body(3)
    config = dict(workload_config(args))
    config["reference_scope"] = REFERENCE_SCOPE
    line = {"metric": METRIC, "value": round(mlups, 3), "unit": UNIT, "n_gpus": args.gpus,
            "steps": timed, "warmup": warm, "ms_per_step": round(dt * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "impl": "reference",
            "config": config,
            "cpu_baseline": {"value": round(mlups, 3), "unit": UNIT, "cores": threads,
                             "kind": kind, "sample": sample},
            "e2e": {"value": round(mlups, 3), "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "with_body_single_level": body}
    if timed < args.steps:
        line["steps_requested"] = args.steps
        line["steps_note"] = ("fewer timed steps than requested: the requested count would exceed the "
                              "120 s budget of the CPU sample")
    print(json.dumps(line), flush=True)


def workload_config(args):
    w = WORKLOAD
    lo, hi = refined_box()
    nf = [2 * (hi[a] - lo[a]) for a in range(3)]
    cells_c = w["nx"] * w["ny"] * w["nz"]
    cells_f = nf[0] * nf[1] * nf[2]
    return {"workload": f"D3Q19 IB-LBM sphere, base grid {w['nx']}x{w['ny']}x{w['nz']} plus 1 refined "
                        f"level (ratio 2) over base cells [{lo[0]},{hi[0]})x[{lo[1]},{hi[1]})x[{lo[2]},{hi[2]}) "
                        f"({nf[0]}x{nf[1]}x{nf[2]} fine cells), D={w['D']:g} base cells, U={w['U']}, "
                        f"Re={w['Re']:g}, golden-spiral markers ~1 fine dx apart, IVC marker IB on the fine "
                        f"level, subcycled (2 fine steps per coarse step), FP32 shifted storage",
            "lattice": "D3Q19", "levels": 2, "coarse_cells": cells_c, "fine_cells": cells_f,
            "updates_per_coarse_step": cells_c + 2 * cells_f, "storage": args.storage,
            "parallelism": f"replicas{args.gpus}",
            "l2_policy": "working set > 1 GB of populations >> 126 MB L2 (no flush needed)"}


def run_single_level(args, world, device):
    """The sphere on its base grid alone (one level, 3,218 markers, stored
    IVC inverse), through ilbm_advance_level with the IB chain overlapped."""
    from ilbmrex_b200 import cases
    from ilbmrex_b200.level import LevelSolver
    w = WORKLOAD
    case, ib, init = cases.sphere(w["nx"], w["ny"], w["nz"], D=w["D"], center=w["center"],
                                  U=w["U"], Re=w["Re"])
    S = LevelSolver(case, args.storage, ib=ib, device=device.index or 0)
    S.set_macro(*init())
    S.step(max(3, args.warmup))
    S.ctx.sync()
    barrier(world)
    K = args.steps
    S.ctx.record(10)
    S.step(K)
    S.ctx.record(11)
    S.ctx.sync()
    t = allreduce_max(S.ctx.elapsed_ms(10, 11), world, device)
    out = {"metric": "MLUPS, the same sphere on its base grid alone (one level)",
           "value": round(world * case.cells * K / (t * 1e-3) / 1e6, 2), "unit": "MLUPS",
           "ms_per_step": round(t / K, 4), "cells": case.cells, "ib_markers": S.num_markers(),
           "steps": K}
    S.close()
    return out


def run_precision(args, world, device):
    """The storage forms of the headline hierarchy against its FP64 run: the
    two-level sphere advanced the same number of coarse steps from the same
    state with FP64, FP32-shifted and FP16-scaled populations; per form its
    ms per coarse step, Cd / Cl and their relative difference to FP64, and
    the relative L2 difference of the fine level's velocity."""
    from ilbmrex_b200.hierarchy import TwoLevelSolver
    tl, ib, init_c, init_f = sphere_hierarchy()
    n = args.precision_steps
    out, ref = {}, None
    for st in ("f64", "f32", "f16"):
        S = TwoLevelSolver(tl, st, ib=ib, device=device.index or 0)
        S.set_macro(init_c(), init_f())
        S.step(n - 1)
        S.ctx.sync()
        S.ctx.record(12)
        S.advance(record_force=True)
        S.ctx.record(13)
        S.ctx.sync()
        ms = S.ctx.elapsed_ms(12, 13)
        u = S.get_macro(1)[1:4]
        cd, cl = float(S.rec[3]), float(S.rec[4])
        S.close()
        if ref is None:
            ref = (u, cd, cl)
            out[st] = {"cd": round(cd, 6), "cl": round(cl, 8), "ms_last_step": round(ms, 3)}
            continue
        du = float(np.sqrt(np.sum((u - ref[0]) ** 2) / np.sum(ref[0] ** 2)))
        out[st] = {"cd": round(cd, 6), "cl": round(cl, 8), "ms_last_step": round(ms, 3),
                   "cd_rel_err_vs_f64": float(f"{abs(cd - ref[1]) / abs(ref[1]):.3e}"),
                   "cl_abs_err_vs_f64": float(f"{abs(cl - ref[2]):.3e}"),
                   "fine_u_rel_l2_vs_f64": float(f"{du:.3e}")}
    return {"what": f"the two-level sphere after {n} coarse steps in each storage form, "
                    "errors against the FP64 run of the same steps (Cl ~ 0 by symmetry: absolute)",
            "steps": n, **out}


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
    ids = [B.add(B.solver(c, ib, init), max_steps=K + 200) for c, ib, init in mix]
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
    # FP32 batched cases against the same cases run alone in FP64 for the
    # same steps: Cd / Cl of the last step
    errs = []
    for idx in range(min(args.batch_check_cases, len(mix))):
        c, ib, init = mix[idx]
        s32 = B.sync(ids[idx])
        cd32, cl32, nsteps = float(s32.rec[3]), float(s32.rec[4]), s32.istep
        R = LevelSolver(c, "f64", ib=ib, device=device.index or 0)
        R.set_macro(*init())
        R.step(nsteps, record_force=True)
        cd64, cl64 = float(R.rec[3]), float(R.rec[4])
        R.close()
        errs.append({"case": c.name, "steps": nsteps, "cd_f32": round(cd32, 6), "cd_f64": round(cd64, 6),
                     "cd_rel_err": float(f"{abs(cd32 - cd64) / max(abs(cd64), 1e-30):.3e}"),
                     "cl_abs_err": float(f"{abs(cl32 - cl64):.3e}")})
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
            "vs_f64_alone": errs,
            "workload": "seeded mix: grids 256x128..1024x512, cylinders D 16-48 Re 20-200, "
                        "NACA0012 pitching (chord 64-128, 2-15 deg, k 0.05-0.3), FP32 storage; "
                        "each case steps through its own IB (stored IVC inverse or CG)"}


def shedding_analysis(cd: np.ndarray, cl: np.ndarray, D: float, U: float, discard: float = 0.25):
    """The acceptance test of the reference's cylinder example
    (Examples/Cylinder_flow/analyze_force.py:62-95, 160-240), restated: drop
    the first quarter of the series; mean Cd; rms Cl, periodic lift when it is
    at least 0.02; Strouhal number from the lift peaks (local maxima at least
    0.4 rms above the mean and 0.4 of the shortest admissible period,
    D / (0.5 U), apart; at least three); Cd in [1.20, 1.80] and, with a
    periodic lift, St in [0.14, 0.20]."""
    n0 = int(len(cd) * discard)
    c_d, c_l = np.asarray(cd[n0:], np.float64), np.asarray(cl[n0:], np.float64)
    cdm, clm = float(np.mean(c_d)), float(np.mean(c_l))
    clr = float(np.sqrt(np.mean((c_l - clm) ** 2)))
    st = None
    if clr > 1e-12:
        min_sep = 0.4 * D / (0.5 * U)
        last = -1e300
        peaks = []
        for i in range(1, len(c_l) - 1):
            if c_l[i] > c_l[i - 1] and c_l[i] >= c_l[i + 1] and c_l[i] - clm >= 0.4 * clr \
                    and i - last >= min_sep:
                peaks.append(i)
                last = i
        if len(peaks) >= 3:
            st = D / (U * float(np.mean(np.diff(peaks))))
    periodic = clr >= 0.02
    return {"samples_used": int(len(c_d)), "cd_mean": round(cdm, 4), "cl_rms": float(f"{clr:.4e}"),
            "periodic_lift": bool(periodic), "strouhal": None if st is None else round(st, 4),
            "match_cd_1.20_1.80": bool(1.2 <= cdm <= 1.8),
            "match_st_0.14_0.20": bool(periodic and st is not None and 0.14 <= st <= 0.20)}


def run_cylinder(args, world, device):
    """The D2Q9 cylinder wake of the 'two AMR levels' configuration: base grid
    1024 x 512, D = 40 base cells centred at (256, 256), inflow U = 0.05,
    Re = 100, max_level = 2 (ratio 2): the finest level over the body and near
    wake (1 R upstream, 4 R downstream, 2 R across plus 6 base cells), the
    middle level around it; the marker IBM on the finest level (markers ~1
    finest dx apart), FP32 storage.  The inflow carries the reference deck's
    transverse velocity 1e-4 (Examples/Cylinder_flow/inputs,
    amrbc.bc_lo_0_uy_val), which breaks the symmetry so that the wake starts
    to shed.  Cell updates per coarse step: coarse cells + 2 x level-1 cells
    + 4 x level-2 cells.  MLUPS over --cyl-steps coarse steps; then the Cd / Cl
    series (time-centred body force, one record per coarse step taken while
    the next step runs) of the configuration's 20,000 coarse steps, continued
    to --cyl-series-steps, each window judged as the reference's
    analyze_force.py judges its run.  Beside it, the reference's CPU level
    step on the same three levels."""
    from ilbmrex_b200 import cases
    from ilbmrex_b200.hierarchy import HierarchySolver
    R, pad, U, D = 20.0, 6.0, 0.05, 40.0
    hc, ib, inits = cases.cylinder_hierarchy(nx=1024, ny=512, D=D, center=(256.0, 256.0), U=U, Re=100.0,
                                             nlev=3, upstream=(R + pad) / D, downstream=(4 * R + pad) / D,
                                             cross=(2 * R + pad) / D, inflow_uy=1.0e-4)
    updates = hc.updates_per_coarse_step()
    # the timed steps replay two coarse steps recorded once as a CUDA graph:
    # the step is 47 launches of a few microseconds each, so per-launch
    # overhead, not bandwidth, bounds it when every launch comes from the host
    S = HierarchySolver(hc, "f32", ib=ib, device=device.index or 0, graphs=True)
    S.set_macro([init() for init in inits])
    S.step(3)
    S.ctx.sync()
    barrier(world)
    K = args.cyl_steps
    l0 = S.ctx.launches()
    S.ctx.record(8)
    S.step(K)
    S.ctx.record(9)
    S.ctx.sync()
    launches = S.ctx.launches() - l0
    graphed = S._graph is not None
    t = allreduce_max(S.ctx.elapsed_ms(8, 9), world, device)
    mlups = world * updates * K / (t * 1e-3) / 1e6
    series = None
    if args.cyl_series_steps > 0:
        # the series restarts from the initial state so that it covers the
        # configuration's whole run
        S.close()
        S = HierarchySolver(hc, "f32", ib=ib, device=device.index or 0)
        S.set_macro([init() for init in inits])
        n = args.cyl_series_steps
        cd, cl = np.zeros(n), np.zeros(n)
        t0 = time.perf_counter()
        for i in range(n):
            S.advance(record_force=True, pipelined=True)
            if i:
                cd[i - 1], cl[i - 1] = S.rec[3], S.rec[4]
        S.flush_records()
        cd[n - 1], cl[n - 1] = S.rec[3], S.rec[4]
        wall = time.perf_counter() - t0
        n20 = min(n, 20000)
        series = {"coarse_steps": int(n), "wall_s": round(wall, 2),
                  "trigger": "inflow transverse velocity 1e-4 (the deck's amrbc.bc_lo_0_uy_val)",
                  "configured_20000_steps": shedding_analysis(cd[:n20], cl[:n20], D, U),
                  "whole_series": shedding_analysis(cd, cl, D, U),
                  "criteria_source": "Examples/Cylinder_flow/analyze_force.py:62-95, 160-240",
                  "cd_every_2000": [round(float(v), 4) for v in cd[1999::2000]],
                  "cl_max_abs_every_2000": [float(f"{np.max(np.abs(cl[k:k + 2000])):.3e}")
                                            for k in range(0, n, 2000)]}
    n_mark = C.c_int64()
    S.L.ilbm_ib_num_markers(S.ib, C.byref(n_mark))
    S.close()
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            levels = [(hc.box_case(l), inits[l], float(2 ** l)) for l in range(hc.nlev)]
            dt, threads, kind, timed = cpu_reference_levels(levels, 5, 3, budget_s=30.0)
            cpu = {"value": round(updates / dt / 1e6, 3), "unit": "MLUPS", "cores": threads, "kind": kind,
                   "sample": f"{timed} level steps of each level after 3 warm-up steps, timed as coarse + "
                             "2 x level 1 + 4 x level 2 per coarse step (the body's forcing, the coarse-fine "
                             "fill and the average-down not included); reference sources compiled in place, "
                             "float, OpenMP"}
        except Exception as e:  # the checker is optional at run time
            cpu = {"value": None, "unit": "MLUPS", "cores": 0, "kind": "port", "sample": f"unavailable: {e}"}
    return {"metric": "MLUPS, D2Q9 cylinder wake 1024x512 with 2 refined levels (max_level 2), FP32",
            "value": round(mlups, 2), "unit": "MLUPS", "ms_per_coarse_step": round(t / K, 4),
            "graph_replay": graphed,
            "levels": [{"box": [list(hc.box_lohi(l)[0][:2]), list(hc.box_lohi(l)[1][:2])],
                        "cells": hc.cells(l)} for l in range(hc.nlev)],
            "updates_per_coarse_step": updates, "steps": K, "gpu_launches": int(launches),
            "ib_markers": int(n_mark.value), "cd_cl_series": series, "cpu_baseline": cpu}


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
    # warm-up (untimed), through the same long-lived server and the plain call:
    # a few short requests of every kind load the kernels and fill the
    # server's memory pools
    wrng = np.random.default_rng(7)
    warm = [make_request(1000 + i, k, wrng, 20, scale=args.serve_scale)
            for i, k in enumerate(["cylinder"] * 4 + ["duct"] * 2 + ["sphere"] * 2)]
    srv = Server("f32", device=device.index or 0, chunk=args.serve_chunk)
    srv.run(warm)
    stats = srv.run(reqs)
    srv.close()
    for r in warm:
        run_alone(r, "f32", device=device.index or 0)
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
            "warmup": f"{len(warm)} requests of 20 steps through the same server and the plain call, untimed",
            "cells_min_max": [int(min(sizes)), int(max(sizes))],
            "steps_min_max": [args.serve_min_steps, args.serve_max_steps],
            "workload": f"seeded Poisson arrivals; 50% D2Q9 cylinder/airfoil (the batched mix's grids), "
                        f"25% D3Q19 duct N x N x 4N (N 32-128), 25% D3Q19 sphere (0.5-1 x 256x128x128); grid "
                        f"edges x {args.serve_scale}; step counts {args.serve_min_steps}-{args.serve_max_steps} "
                        f"(the served configuration asks 1000-20000: the upper part is cut so the run "
                        f"fits the bench's time)",
            "plain_arm": "each request alone through ilbm_advance_level, steps queued back to back with "
                         "the force record of every step copied to pinned memory in stream order, one "
                         "synchronisation per request"}


def level_step_ms(L, ctx, box, params, K: int) -> float:
    """Mean device time (CUDA events on the library stream) of K launches of
    ilbm_level_step on one box, after two untimed ones; the box's f_in is
    read and its f_out written each time, so the state is left as it was."""
    from ilbmrex_b200 import capi
    for r in range(K + 2):
        if r >= 2:
            ctx.record(16 + 2 * (r - 2))
        capi.check(L.ilbm_level_step(ctx.h, C.byref(box), 1, C.byref(params)), "level step")
        if r >= 2:
            ctx.record(17 + 2 * (r - 2))
    ctx.sync()
    return float(np.mean([ctx.elapsed_ms(16 + 2 * r, 17 + 2 * r) for r in range(K)]))


def run_roofline_only(args):
    """The dominant kernel alone, for profiling: the level step of the
    sphere's 256 x 128 x 128 base level (no body, the headline's storage
    form, the library's population layout) launched --steps times after
    --warmup level steps; prints one JSON line with its roofline figures."""
    import torch
    from ilbmrex_b200 import cases
    from ilbmrex_b200.level import LevelSolver
    w = WORKLOAD
    case, _, init = cases.sphere(w["nx"], w["ny"], w["nz"], D=w["D"], center=w["center"], U=w["U"],
                                 Re=w["Re"])
    S = LevelSolver(case, args.storage, ib=None)
    S.set_macro(*init())
    S.step(max(3, args.warmup))
    S.ctx.sync()
    sbytes = {"f64": 8, "f32": 4, "f16": 2}[args.storage]
    B_cell = 2 * case.lattice.q * sbytes
    ms = level_step_ms(S.L, S.ctx, S._box(S.f, S.f_next), S.params, max(1, args.steps))
    peak, kind = peaks()
    achieved = B_cell * case.cells / (ms * 1e-3) / 1e9
    print(json.dumps({"roofline_only": True, "kernel": f"k_step<D3Q{case.lattice.q},{args.storage}>",
                      "cells": case.cells, "bytes_per_cell": B_cell, "kernel_ms": round(ms, 4),
                      "achieved_gbs": round(achieved, 1), "peak_gbs": peak, "peak_source": kind,
                      "frac": round(achieved / peak, 4), "launches": max(1, args.steps) + 2}), flush=True)
    S.close()
    torch.cuda.synchronize()


def run_b200(args):
    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    from ilbmrex_b200 import capi, cases
    from ilbmrex_b200.level import LevelSolver

    if args.only_batched or args.only_served or args.only_cylinder:  # profiling aids: one workload alone
        if args.only_cylinder:
            out = run_cylinder(args, world, device)
        else:
            out = run_batched(args, world, device) if args.only_batched else run_served(args, world, device)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return

    from ilbmrex_b200.hierarchy import TwoLevelSolver
    tl, ib, init_c, init_f = sphere_hierarchy()
    S = TwoLevelSolver(tl, args.storage, ib=ib, device=local)
    S.set_macro(init_c(), init_f())
    ctx = S.ctx
    cells_c = tl.coarse.cells
    cells_f = int(np.prod(tl.fine_n_cell))
    updates = cells_c + 2 * cells_f
    q = tl.coarse.lattice.q
    sbytes = {"f64": 8, "f32": 4, "f16": 2}[args.storage]
    B_cell = 2 * q * sbytes

    # ---- device-resident timed region: K coarse steps --------------------
    K = args.steps
    ctx.sync()
    ctx.record(2)
    S.advance()  # includes the one-time CSR build of the IVC operator
    ctx.record(3)
    ctx.sync()
    first_step_ms = ctx.elapsed_ms(2, 3)
    for _ in range(max(3, args.warmup) - 1):
        S.advance()
    ctx.sync()
    torch.cuda.synchronize(device)
    launches0 = ctx.launches()
    sampler = ClockSampler(local)
    with sampler:
        barrier(world)
        ctx.sync()
        ctx.record(0)
        for _ in range(K):
            S.advance()
        ctx.record(1)
        ctx.sync()
        barrier(world)
    launches = ctx.launches() - launches0
    t_ms = ctx.elapsed_ms(0, 1)
    value, t_max = aggregate_mlups(updates, K, t_ms, world, device)
    clocks = sampler.summary()

    # ---- roofline pass: the dominant kernel, the level step k_step
    # <D3Q19, storage> with its ghost-shell push, on the coarse level
    # (4,194,304 cells), from the current state into the scratch buffer (the
    # hierarchy's state is left as it was) ------------------------------------
    Cl = S.C
    kern_ms = level_step_ms(S.L, ctx, Cl.box(Cl.f, Cl.f_next), S.pc, max(3, min(K, 20)))
    peak, peak_kind = peaks()
    achieved = B_cell * cells_c / (kern_ms * 1e-3) / 1e9
    # the same kernel on the fine level as the hierarchy runs it (caller-filled
    # ghosts, the body's force arrays on its band)
    Fl = S.F
    fine_ms = level_step_ms(S.L, ctx, Fl.box(Fl.f, Fl.f_next, force=Fl.fa, force_prev=Fl.fb), S.pf,
                            max(3, min(K, 20)))
    fine_achieved = B_cell * cells_f / (fine_ms * 1e-3) / 1e9

    n_mark = C.c_int64()
    S.L.ilbm_ib_num_markers(S.ib, C.byref(n_mark))
    cg_it = C.c_int()
    S.L.ilbm_ib_solver_stats(S.ib, C.byref(cg_it))
    S.close()

    # ---- end-to-end through the public call: per coarse step the host
    # parameter structs go down and the force record (Eulerian and marker
    # force sums, status) comes back to pinned host memory; the host takes
    # each step's record (Cd / Cl) after queueing the next step.  A fresh
    # hierarchy from the same initial state and the same warm-up steps, so
    # that this leg times the same coarse steps of the flow as the
    # device-timed one (the body's CG needs more iterations as the wake
    # develops) ---------------------------------------------------------------
    Ke = max(3, K)  # as many steps as the device-timed region: start-up and the last record amortised
    S = TwoLevelSolver(tl, args.storage, ib=ib, device=local)
    S.set_macro(init_c(), init_f())
    for _ in range(max(3, args.warmup)):
        S.advance()
    S.ctx.sync()
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(Ke):
        S.advance(record_force=True, pipelined=True)
    S.flush_records()
    S.ctx.sync()
    e2e_s = allreduce_max(time.perf_counter() - t0, world, device)
    e2e = world * updates * Ke / e2e_s / 1e6
    h2d = 2 * C.sizeof(capi.LevelParams_t) + 2 * C.sizeof(capi.Box_t) + 24
    d2h = 8 * 8
    cd, cl = float(S.rec[3]), float(S.rec[4])

    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get("k_step_d3q19_f32_bytes_per_launch")
        except Exception:
            traffic = None
    S.close()

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            mlups, dt, threads, kind, timed, sample = cpu_reference_steps(2, 3)
            cpu_base = {"value": round(mlups, 3), "unit": UNIT, "cores": threads, "kind": kind,
                        "sample": sample, "scope": REFERENCE_SCOPE}
        except Exception as e:  # the checker is optional at run time
            cpu_base = {"value": None, "unit": UNIT, "cores": 0, "kind": "port",
                        "sample": f"unavailable: {e}"}

    single = None if args.no_single_level else run_single_level(args, world, device)
    precision = None if args.no_precision else run_precision(args, world, device)
    batched = None
    if not args.no_batched:
        batched = run_batched(args, world, device)
    served = None
    if not args.no_served:
        served = run_served(args, world, device)
    cylinder = None
    if not args.no_cylinder:
        cylinder = run_cylinder(args, world, device)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world,
            "steps": K, "warmup": max(3, args.warmup), "ms_per_step": round(t_max / K, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage != "f64" else "f64", "data": "synthetic",
            "config": workload_config(args),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": "level step = k_step<D3Q19,F32_SHIFT> (ghost-shell push in its "
                                   "leading blocks), timed alone on the 256x128x128 coarse level",
                         "kernel_ms": round(kern_ms, 4), "bytes_per_cell": B_cell,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6650 GB/s",
                         "fine_level": {"kernel_ms": round(fine_ms, 4), "cells": cells_f,
                                        "achieved": round(fine_achieved, 1),
                                        "frac": round(fine_achieved / peak, 4),
                                        "what": "k_step on the 192x128x128 fine box (caller-filled "
                                                "ghosts, body force arrays on its band)"}},
            "cpu_baseline": cpu_base,
            "e2e": {"value": round(e2e, 2), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "ib_markers": int(n_mark.value),
            "ivc_cg_iterations": int(cg_it.value),
            "cd_cl_after": [round(cd, 5), round(cl, 6)],
            "first_step_ms_incl_ivc_setup": round(first_step_ms, 2),
            "precision": precision,
            "single_level": single,
            "batched": batched,
            "served": served,
            "cylinder_three_levels": cylinder,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f64", "f32", "f16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=0, help="sphere level size override (tests)")
    ap.add_argument("--ny", type=int, default=0)
    ap.add_argument("--nz", type=int, default=0)
    ap.add_argument("--no-batched", action="store_true", help="skip the batched workload")
    ap.add_argument("--no-single-level", action="store_true", help="skip the single-level sphere")
    ap.add_argument("--no-precision", action="store_true", help="skip the storage-form error check")
    ap.add_argument("--precision-steps", type=int, default=200)
    ap.add_argument("--no-served", action="store_true", help="skip the served workload")
    ap.add_argument("--no-cylinder", action="store_true", help="skip the three-level cylinder workload")
    ap.add_argument("--cyl-steps", type=int, default=200, help="timed coarse steps of the cylinder")
    ap.add_argument("--cyl-series-steps", type=int, default=60000,
                    help="coarse steps of the cylinder's Cd / Cl series (0: none)")
    ap.add_argument("--only-cylinder", action="store_true",
                    help="run only the three-level cylinder workload and print its result (profiling aid)")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-rate", type=float, default=200.0, help="arrivals per second")
    ap.add_argument("--serve-scale", type=float, default=1.0)
    ap.add_argument("--serve-min-steps", type=int, default=1000)
    ap.add_argument("--serve-max-steps", type=int, default=2000)
    ap.add_argument("--serve-chunk", type=int, default=100)
    ap.add_argument("--only-batched", action="store_true",
                    help="run only the batched workload and print its result (profiling aid)")
    ap.add_argument("--only-served", action="store_true",
                    help="run only the served workload and print its result (profiling aid)")
    ap.add_argument("--batch-cases", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=40)
    ap.add_argument("--batch-plain-steps", type=int, default=8)
    ap.add_argument("--batch-check-cases", type=int, default=4)
    ap.add_argument("--roofline-only", action="store_true",
                    help="time only the level step of the sphere's base level (profiling aid)")
    args = ap.parse_args()
    if args.nx:
        set_workload_size(args.nx, args.ny or args.nx // 2, args.nz or args.nx // 2)
    if args.impl == "reference":
        run_reference(args)
    elif args.roofline_only:
        run_roofline_only(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
