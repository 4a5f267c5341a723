"""Host mirror of the batch engine (``ilbm_batch_*`` in ``include/ilbm_b200.h``).

Many independent single-level cases of one lattice and storage form advance
together on one GPU: one launch per immersed-boundary stage for all cases,
one persistent collide-stream kernel over every case's cells, two steps per
CUDA-graph replay.  Each case is a :class:`~ilbmrex_b200.level.LevelSolver`
built on the batch's context; it takes its first step on its own (the step
that reads the stored macro fields and builds the IVC operator, as the
reference's first AdvancePhiAtLevel does) and then joins.  While a case is
in the batch its state lives in the solver's buffers; :meth:`Batch.sync`
hands it back to the solver (buffer roles, time, step count).

No counterpart in the reference, which advances one case per run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .level import Context, LevelSolver


class Batch:
    def __init__(self, lattice, storage: str = "f32", device: int = 0, rec_slots: int = 256):
        self.ctx = Context(lattice, storage, device)
        self.L = self.ctx.L
        self.storage = storage
        self.device = device
        h = C.c_void_p()
        capi.check(self.L.ilbm_batch_create(self.ctx.h, int(rec_slots), C.byref(h)), "batch_create")
        self.h = h
        self.members: dict[int, LevelSolver] = {}
        self._taken: dict[int, int] = {}  # records already folded into the solver

    # ---- composition ------------------------------------------------------
    def solver(self, case, ib=None, init=None) -> LevelSolver:
        """A LevelSolver on the batch's context (initialised from init())."""
        s = LevelSolver(case, self.storage, ib=ib, device=self.device, ctx=self.ctx)
        if init is not None:
            s.set_macro(*init())
        return s

    def add(self, s: LevelSolver, max_steps: int) -> int:
        """Joins a solver to the batch (after its first step, or its first step
        since a restart when it has a body, taken here if needed); returns the
        case id."""
        if s.ctx is not self.ctx:
            raise capi.IlbmError("the solver must be built on the batch's context (Batch.solver)")
        if s.istep == 0 or (s.ib is not None and not s.ib_ready):
            s.advance_phi_at_level(record_force=s.ib is not None)
        b = s._box(s.f, s.f_next, force=s.force_cur if s.ib is not None else None,
                   force_prev=s.force_prev if s.ib is not None else None)
        cid = C.c_int()
        capi.check(self.L.ilbm_batch_add(self.h, C.byref(b), C.byref(s.params), s.ib, s.case.dt,
                                         s.time, int(max_steps), C.byref(cid)), "batch_add")
        self.members[cid.value] = s
        self._taken[cid.value] = 0
        s._batch_bufs = (s.f, s.f_next, s.force_cur, s.force_prev)  # the box as added
        return cid.value

    def remove(self, cid: int) -> LevelSolver:
        """Hands the case's state back to its solver and drops it."""
        s = self.sync(cid)
        capi.check(self.L.ilbm_batch_remove(self.h, int(cid)), "batch_remove")
        del self.members[cid]
        del self._taken[cid]
        return s

    # ---- stepping ---------------------------------------------------------
    def step(self, n: int = 1):
        capi.check(self.L.ilbm_batch_step(self.h, int(n)), "batch_step")

    def tune(self, trial_steps: int = 6):
        w, cps, ms = C.c_int(), C.c_int(), C.c_float()
        capi.check(self.L.ilbm_batch_tune(self.h, int(trial_steps), C.byref(w), C.byref(cps),
                                          C.byref(ms)), "batch_tune")
        return w.value, cps.value, ms.value

    def set_tiles(self, tile_w: int, ctas_per_sm: int = 0):
        capi.check(self.L.ilbm_batch_set_tiles(self.h, int(tile_w), int(ctas_per_sm)), "batch_set_tiles")

    def progress(self) -> dict[int, tuple[int, int]]:
        """case id -> (steps taken in the batch, steps remaining); one sync."""
        n = C.c_int()
        capi.check(self.L.ilbm_batch_progress(self.h, 0, None, None, None, C.byref(n)), "batch_progress")
        m = n.value
        ids = (C.c_int * max(m, 1))()
        done = (C.c_int64 * max(m, 1))()
        left = (C.c_int * max(m, 1))()
        capi.check(self.L.ilbm_batch_progress(self.h, m, ids, done, left, C.byref(n)), "batch_progress")
        return {ids[i]: (done[i], left[i]) for i in range(m)}

    def size(self):
        n, cells = C.c_int(), C.c_int64()
        capi.check(self.L.ilbm_batch_size(self.h, C.byref(n), C.byref(cells)), "batch_size")
        return n.value, cells.value

    # ---- results ----------------------------------------------------------
    def records(self, cid: int) -> np.ndarray:
        """Per-step (Eulerian force sum (3), marker force sum (3)) of the case
        since it joined, oldest first."""
        n = C.c_int()
        capi.check(self.L.ilbm_batch_records(self.h, int(cid), None, 0, C.byref(n)), "batch_records")
        out = np.zeros(max(n.value, 1) * 6)
        capi.check(self.L.ilbm_batch_records(self.h, int(cid), out.ctypes.data_as(C.POINTER(C.c_double)),
                                             n.value, C.byref(n)), "batch_records")
        return out[:n.value * 6].reshape(n.value, 6)

    def sync(self, cid: int) -> LevelSolver:
        """Brings the solver up to date with the case (buffer roles, time,
        step count, force record of the last step; every step's record is
        appended to ``solver.rec_history`` when the solver has that list)."""
        s = self.members[cid]
        par, steps, t = C.c_int(), C.c_int64(), C.c_double()
        capi.check(self.L.ilbm_batch_case_state(self.h, int(cid), C.byref(par), C.byref(steps),
                                                C.byref(t)), "batch_case_state")
        new = steps.value - self._taken[cid]
        if new > 0:
            if s.ib is not None:
                hist = getattr(s, "rec_history", None)
                raw = np.asarray(self.records(cid)[self._taken[cid]:steps.value], dtype=np.float64)
                if len(raw):
                    recs = s.force_records(raw[:, 0:3], raw[:, 3:6])
                    s.rec = recs[-1].copy()
                    if hist is not None:
                        hist.extend(recs)
            s.istep += new
            self._taken[cid] = steps.value
        # parity 0: the state is in the buffers as added; 1: roles swapped
        f0, f1, fc, fp = s._batch_bufs
        if par.value == 0:
            s.f, s.f_next, s.force_cur, s.force_prev = f0, f1, fc, fp
        else:
            s.f, s.f_next, s.force_cur, s.force_prev = f1, f0, fp, fc
        s.time = t.value
        return s

    def close(self):
        if self.h is not None:
            self.L.ilbm_batch_destroy(self.h)
            self.h = None
        for s in self.members.values():
            s.close()
        self.members = {}
        if self.ctx is not None:
            self.ctx.close()
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
