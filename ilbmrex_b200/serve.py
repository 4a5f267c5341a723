"""Serving loop: continuous batching of LBM solve requests on one GPU.

A request is one single-level case (D2Q9 cylinder or pitching airfoil, D3Q19
square duct or sphere) and a step count.  Requests arrive over time; the
server admits them first-come first-served while their device footprint fits
the HBM budget, keeps their populations, forces and markers resident, and
advances every admitted case together: one batch engine per lattice (each
on its own stream, so D2Q9 and D3Q19 work overlaps on the device), stepped
in chunks, with cases joining and leaving between chunks.  A finished case
returns its per-step force record (Cd, Cl of an immersed body) or its mean
velocity, and its latency (completion minus arrival).  The run reports p50 /
p99 latency and aggregate MLUPS.

No counterpart in the reference, which runs one case per process.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import cases as C
from .batch import Batch
from .lattice import D2Q9, D3Q19
from .level import LevelSolver


@dataclass
class Request:
    rid: int
    kind: str                 # "cylinder", "airfoil", "duct" or "sphere"
    case: C.LevelCase
    ib: C.MarkerIB | None
    init: object
    steps: int
    arrival: float = 0.0      # seconds after the start of the run
    # filled by the server
    admitted: float | None = None
    finished: float | None = None
    cd_cl: np.ndarray | None = None   # (steps, 2) for bodies: Cd, Cl per step
    mean_u: np.ndarray | None = None  # mean velocity at completion
    f_final: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return (self.finished - self.arrival) if self.finished is not None else float("nan")


def make_request(rid: int, kind: str, rng: np.random.Generator, steps: int, scale: float = 1.0) -> Request:
    """A request of the served mix with seeded parameters.  scale < 1 shrinks
    grid edges (the sizes of the served configuration span 1e5-3e7 cells)."""
    if kind in ("cylinder", "airfoil"):
        (case, ib, init), = C.batch_mix(1, seed=int(rng.integers(1 << 30)))
        if scale != 1.0:
            nx = max(64, int(case.n_cell[0] * scale) // 8 * 8)
            ny = max(48, int(case.n_cell[1] * scale) // 8 * 8)
            if ib.geometry_type == 2:
                chord = max(16.0, min(ib.airfoil[0] * scale, 0.45 * nx, 0.9 * ny))
                case, ib, init = C.pitching_airfoil(nx=nx, ny=ny, chord=chord,
                                                    pivot=(0.25 * nx + 0.37, 0.5 * ny - 0.21),
                                                    amplitude_deg=math.degrees(ib.airfoil[3]),
                                                    reduced_frequency=ib.airfoil[4] * 2 * math.pi * chord / (2 * ib.U0))
            else:
                D = max(8.0, min(2.0 * ib.R * scale, 0.3 * ny))
                case, ib, init = C.cylinder(nx=nx, ny=ny, D=D, center=(0.25 * nx + 0.37, 0.5 * ny - 0.21),
                                            U=ib.U0, Re=float(rng.uniform(20.0, 200.0)))
        kind = "airfoil" if ib.geometry_type == 2 else "cylinder"
    elif kind == "duct":
        N = int(rng.integers(32, 129))
        N = max(8, int(N * scale))
        case, init = C.square_duct(N=N, L=4 * N, force=1.0e-5, nu=0.06)
        ib = None
    elif kind == "sphere":
        s = float(rng.uniform(0.5, 1.0)) * scale
        nx, ny = max(32, int(256 * s) // 8 * 8), max(16, int(128 * s) // 8 * 8)
        D = 32.0 * s
        case, ib, init = C.sphere(nx, ny, ny, D=D, center=(0.25 * nx + 0.31, 0.5 * ny - 0.17, 0.5 * ny + 0.13),
                                  U=0.04, Re=100.0)
    else:
        raise ValueError(kind)
    return Request(rid, kind, case, ib, init, int(steps))


class Server:
    """Continuous-batching server (FP32 storage by default)."""

    def __init__(self, storage: str = "f32", device: int = 0, chunk: int = 50,
                 hbm_budget: int | None = None):
        self.storage = storage
        self.device = device
        self.chunk = int(chunk)
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = int(0.8 * free)
        self.budget = int(hbm_budget)
        self.used = 0
        self.batches: dict[int, Batch] = {}
        self.active: dict[int, tuple] = {}   # rid -> (q, cid, request, solver, footprint)

    def _batch(self, lattice) -> Batch:
        if lattice.q not in self.batches:
            self.batches[lattice.q] = Batch(lattice, self.storage, device=self.device, rec_slots=1024)
        return self.batches[lattice.q]

    @staticmethod
    def footprint(req: Request, storage: str) -> int:
        s = {"f64": 8, "f32": 4, "f16": 2}[storage]
        r = 8 if storage == "f64" else 4
        nx, ny, nz = req.case.n_cell
        d = req.case.dim
        gf = (nx + 2) * (ny + 2) * ((nz + 2) if d == 3 else 1)
        gm = (nx + 4) * (ny + 4) * ((nz + 4) if d == 3 else 1)
        n = 2 * req.case.lattice.q * gf * s + 10 * gm * r
        if req.ib is not None:
            from .level import ib_footprint
            n += ib_footprint(req.case, req.ib)
        return int(n)

    def _admit(self, req: Request, now: float) -> bool:
        fp = self.footprint(req, self.storage)
        if self.used + fp > self.budget and self.active:
            return False
        B = self._batch(req.case.lattice)
        S = B.solver(req.case, req.ib, req.init)
        cid = B.add(S, max_steps=req.steps - 1)  # takes the request's first step itself
        req.admitted = now
        self.used += fp
        self.active[req.rid] = (req.case.lattice.q, cid, req, S, fp)
        if req.ib is not None:
            S.rec_history = [S.rec.copy()]  # the first step's record
        return True

    def _retire(self, rid: int, now: float):
        q, cid, req, S, fp = self.active.pop(rid)
        self.batches[q].remove(cid)  # hands the state and force records back
        if req.ib is not None:
            req.cd_cl = np.array([r[3:5] for r in S.rec_history])
        req.mean_u = S.mean_velocity()
        req.f_final = None
        req.finished = now
        S.close()
        self.used -= fp

    def run(self, requests: list[Request], keep_f: bool = False) -> dict:
        """Serves the requests (their .arrival set) and returns the statistics."""
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: list[Request] = []
        t0 = time.perf_counter()
        lups_done: dict[int, int] = {}
        spent = {"admit": 0.0, "step": 0.0, "retire": 0.0, "idle": 0.0}
        while pending or queue or self.active:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                queue.append(pending.pop(0))
            ta = time.perf_counter()
            while queue and self._admit(queue[0], now):
                r = queue.pop(0)
                lups_done[r.rid] = r.case.cells  # its first step
            spent["admit"] += time.perf_counter() - ta
            if not self.active:
                if pending:
                    ti = time.perf_counter()
                    time.sleep(max(0.0, min(0.01, pending[0].arrival - now)))
                    spent["idle"] += time.perf_counter() - ti
                continue
            ts = time.perf_counter()
            # next chunk: every batch advances `chunk` steps; a case that
            # reaches its step count stops there on the device and sits out
            for q, B in self.batches.items():
                if any(v[0] == q for v in self.active.values()):
                    B.step(self.chunk)  # asynchronous: the lattices' batches overlap
            finished = []
            for q, B in self.batches.items():
                if not any(v[0] == q for v in self.active.values()):
                    continue
                prog = B.progress()  # synchronises this batch
                for rid, v in self.active.items():
                    if v[0] == q:
                        done, left = prog[v[1]]
                        if left == 0:
                            finished.append(rid)
                        lups_done[rid] = v[2].case.cells * (1 + done)
            spent["step"] += time.perf_counter() - ts
            now = time.perf_counter() - t0
            tr = time.perf_counter()
            for rid in finished:
                req = self.active[rid][2]
                if keep_f:
                    S = self.batches[self.active[rid][0]].sync(self.active[rid][1])
                    req.f_final = S.get_f()
                    f_keep = req.f_final
                else:
                    f_keep = None
                self._retire(rid, now)
                req.f_final = f_keep
            spent["retire"] += time.perf_counter() - tr
        makespan = time.perf_counter() - t0
        lups = sum(lups_done.values())
        lat = np.array([r.latency for r in requests])
        return {"requests": len(requests), "makespan_s": makespan,
                "mlups": lups / makespan / 1e6,
                "p50_latency_s": float(np.percentile(lat, 50)),
                "p99_latency_s": float(np.percentile(lat, 99)),
                "lattice_updates": int(lups),
                "time_s": {k: round(v, 4) for k, v in spent.items()}}

    def close(self):
        for v in list(self.active.values()):
            v[3].close()
        self.active = {}
        for B in self.batches.values():
            B.close()
        self.batches = {}


def run_alone(req: Request, storage: str = "f32", device: int = 0, keep_f: bool = False) -> Request:
    """The same request through the plain single-case call, for comparison:
    its steps queued back to back through ilbm_advance_level, each step's
    force record copied to pinned memory in stream order and read once at
    the end (LevelSolver.run_recorded)."""
    S = LevelSolver(req.case, storage, ib=req.ib, device=device)
    S.set_macro(*req.init())
    recs = S.run_recorded(req.steps)
    out = Request(req.rid, req.kind, req.case, req.ib, req.init, req.steps, req.arrival)
    out.cd_cl = recs[:, 3:5].copy() if req.ib is not None else None
    out.mean_u = S.mean_velocity()
    out.f_final = S.get_f() if keep_f else None
    S.close()
    return out


def poisson_arrivals(n: int, rate: float, rng: np.random.Generator) -> np.ndarray:
    """n arrival times (seconds) of a Poisson process of the given rate."""
    return np.cumsum(rng.exponential(1.0 / rate, size=n)) - 0.0
