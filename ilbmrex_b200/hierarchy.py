"""Static hierarchies on the GPU through the C ABI.

``HierarchySolver`` holds a coarse level equal to the domain and one fixed
box on each finer level (refinement ratio 2, ``cases.HierarchyCase``) in
device memory and advances them with ``ilbm_advance_hierarchy``: a level's
step, two substeps of the next finer level whose ghost cells come from this
level's macro fields on the device, then average-down, recursively
(AmrCoreLBM::timeStepWithSubcycling, Source/Core/AmrCoreLBM.cpp:1690-1755,
without regrid).  ``TwoLevelSolver`` is the two-level case advanced by
``ilbm_advance_two_level``, whose schedule overlaps the coarse step with the
fine level's body forcing.  A marker body lives on the finest level
(Source/Core/AdvanceLBMAtLevel.cpp:30, 73-93).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import capi
from .cases import HierarchyCase, MarkerIB, TwoLevelCase
from .level import (_REAL_DT, _TORCH_DT, Context, LevelSolver, alloc_populations, ib_params,
                    level_geom, level_params)


class _Level:
    """Device buffers of one level box: populations and stored macro fields
    in pairs, forces in a pair (fine level with a body)."""

    def __init__(self, q, dim, n_cell, lo, storage, dev, with_force):
        self.dim, self.lo = dim, tuple(lo)
        self.n_cell = tuple(n_cell)
        self.gf, self.gm = 1, 2
        nx, ny, nz = n_cell
        gz_f = nz + 2 * self.gf if dim == 3 else 1
        gz_m = nz + 2 * self.gm if dim == 3 else 1
        fdt, rdt = _TORCH_DT[storage], _REAL_DT[storage]
        fsh = (q, gz_f, ny + 2 * self.gf, nx + 2 * self.gf)
        msh = (gz_m, ny + 2 * self.gm, nx + 2 * self.gm)
        self.f = alloc_populations(*fsh, fdt, dev, ngrow=self.gf)
        self.f_next = alloc_populations(*fsh, fdt, dev, ngrow=self.gf)
        self.m = torch.zeros((4,) + msh, dtype=rdt, device=dev)
        self.m_next = torch.zeros((4,) + msh, dtype=rdt, device=dev)
        self.fa = torch.zeros((3,) + msh, dtype=rdt, device=dev) if with_force else None
        self.fb = torch.zeros((3,) + msh, dtype=rdt, device=dev) if with_force else None

    def box(self, f_in=None, f_out=None, m_in=None, m_out=None, force=None, force_prev=None):
        b = capi.Box_t()
        for d in range(3):
            b.lo[d] = self.lo[d] if d < self.dim else 0
            b.hi[d] = self.lo[d] + self.n_cell[d] - 1 if d < self.dim else 0
        b.ngrow_f, b.ngrow_m = self.gf, self.gm
        fs, ms = self.f.stride(), self.m.stride()
        b.fstride[0], b.fstride[1], b.fstride[2] = fs[2], fs[1], fs[0]
        b.mstride[0], b.mstride[1], b.mstride[2] = ms[2], ms[1], ms[0]
        ptr = lambda t: t.data_ptr() if t is not None else None
        b.f_in, b.f_out = ptr(f_in), ptr(f_out)
        b.macro_in, b.macro_out = ptr(m_in), ptr(m_out)
        b.force, b.force_prev = ptr(force), ptr(force_prev)
        return b

    def valid(self, t, g):
        nx, ny, nz = self.n_cell
        if self.dim == 3:
            return t[..., g:g + nz, g:g + ny, g:g + nx]
        return t[..., :, g:g + ny, g:g + nx]


class HierarchySolver:
    """A static hierarchy (``cases.HierarchyCase``: coarse level = the domain,
    one box per finer level, ratio 2) stepped on the GPU through
    ``ilbm_advance_hierarchy``; a marker body lives on the finest level."""

    def __init__(self, hc: HierarchyCase, storage: str = "f64", ib: MarkerIB | None = None,
                 device: int = 0, f16_scale: float = 1024.0, graphs: bool = False):
        """graphs: step(n) replays two coarse steps recorded once as a CUDA
        graph (``ilbm_graph_*``) instead of issuing every launch from the
        host, when the body (if any) does not move and the step is not the
        first after initialisation; the results are those of the same steps
        taken one call at a time."""
        if not torch.cuda.is_available():
            raise capi.IlbmError("HierarchySolver needs a CUDA device")
        self.use_graphs = graphs
        self._graph = None
        self._graph_failed = False
        self.hc = hc
        self.nlev = hc.nlev
        self.storage = storage
        self.dev = torch.device("cuda", device)
        c = hc.coarse
        top = hc.nlev - 1
        self.case = hc.level_case(top)          # the finest level (force record, body)
        self.ib_case = ib
        self.dim = c.dim
        self.ctx = Context(c.lattice, storage, device)
        self.L = self.ctx.L
        q = c.lattice.q
        self.levels = []
        self.params = []
        self._lb = []
        for l in range(hc.nlev):
            lo, _ = hc.box_lohi(l)
            self.levels.append(_Level(q, c.dim, hc.n_cell_of(l), lo, storage, self.dev,
                                      ib is not None and l == top))
            if l == 0:
                p = level_params(c, uniform_force=True, f16_scale=f16_scale)
            else:
                p = level_params(hc.level_case(l), uniform_force=(ib is None or l < top),
                                 f16_scale=f16_scale)
                p.ghost_mode = capi.GHOST_CALLER
                lo, hi = hc.box_lohi(l)
                lb = (C.c_int * 6)(*lo, *hi)
                self._lb.append(lb)
                p.level_boxes = C.cast(lb, C.POINTER(C.c_int))
                p.nlevel_boxes = 1
            self.params.append(p)
        self.C, self.F = self.levels[0], self.levels[top]
        self.pc, self.pf = self.params[0], self.params[top]
        self.ib = None
        if ib is not None:
            self._geom = level_geom(self.case)
            self._ibp = ib_params(ib, self.dim)
            h = C.c_void_p()
            capi.check(self.L.ilbm_ib_create(self.ctx.h, C.byref(self._ibp), C.byref(self._geom),
                                             C.byref(h)), "ilbm_ib_create")
            self.ib = h
            lo, hi = (C.c_int * 3)(), (C.c_int * 3)()
            capi.check(self.L.ilbm_ib_force_region(self.ib, lo, hi), "ib_force_region")
            self.force_region = (tuple(lo), tuple(hi))
            for d in range(3):
                self.pf.force_lo[d], self.pf.force_hi[d] = lo[d], hi[d]
        self.time = 0.0
        self.istep = 0
        self.first_step = True
        self.have_prev_body = False
        self.prev_body = np.zeros(3)
        self.rec = np.zeros(18)
        # pipelined force records: two pinned host slots, the pending one
        self._rec_bufs = None
        self._rec_slot = 0
        self._pending = None

    # ---- initialisation (MakeNewLevelFromScratch per level + InitData) ----
    def set_macro(self, *inits):
        """Initial (rho, u, v, w) of each level on its valid cells, coarsest
        first (one argument per level, or one list of them); each level's
        populations become their equilibrium, then every level is averaged
        down onto the one above, finest first (InitData,
        AmrCoreLBM.cpp:704-722)."""
        if len(inits) == 1 and len(inits[0]) == self.nlev and not isinstance(inits[0][0], np.ndarray):
            inits = tuple(inits[0])
        for lvl, vals in zip(self.levels, inits):
            v = lvl.valid(lvl.m, lvl.gm)
            for n in range(4 if self.dim == 3 else 3):
                v[n].copy_(torch.as_tensor(np.asarray(vals[n]), dtype=lvl.m.dtype))
            torch.cuda.synchronize(self.dev)
            b = lvl.box(lvl.f, lvl.f_next, m_in=lvl.m)
            capi.check(self.L.ilbm_init_equilibrium(self.ctx.h, C.byref(b)), "init_equilibrium")
        for l in range(self.nlev - 1, 0, -1):
            crs, fin = self.levels[l - 1], self.levels[l]
            bc = crs.box(crs.f, None, m_in=crs.m)
            bf = fin.box(fin.f, None, m_in=fin.m)
            capi.check(self.L.ilbm_average_down(self.ctx.h, C.byref(bc), C.byref(self.params[l - 1]),
                                                C.byref(bf), C.byref(self.params[l])), "average_down")
        self.ctx.sync()
        self.time, self.istep = 0.0, 0
        self.first_step = True

    # ---- one coarse step ---------------------------------------------------
    def _launch_step(self, record_into=None):
        top = self.nlev - 1
        arr = (capi.Box_t * self.nlev)()
        for l, lvl in enumerate(self.levels):
            if l < top:
                arr[l] = lvl.box(lvl.f, lvl.f_next, m_in=lvl.m, m_out=lvl.m_next)
            else:
                arr[l] = lvl.box(lvl.f, lvl.f_next, m_in=lvl.m if self.first_step else None,
                                 force=lvl.fa, force_prev=lvl.fb)
        pa = (capi.LevelParams_t * self.nlev)(*self.params)
        flags = capi.HIERARCHY_FIRST_STEP if self.first_step else 0
        capi.check(self.L.ilbm_advance_hierarchy(self.ctx.h, self.nlev, arr, pa, self.ib,
                                                 self.hc.coarse.dt, self.time, flags),
                   "advance_hierarchy")

    def advance(self, record_force: bool = False, pipelined: bool = False):
        """One coarse step.  record_force: the force record (self.rec) of the
        step; pipelined: its sums are copied to the host without waiting, and
        the record of the previous step is taken instead (flush_records takes
        the last one), so the next step is queued before the host waits.
        Where the solver can take the record with the step itself
        (TwoLevelSolver), the pipelined record runs beside the step's end."""
        fused = record_force and pipelined and self.ib is not None and self._records_with_step()
        buf = self._next_rec_buf() if fused else None
        self._launch_step(record_into=buf)
        Cl = self.C
        Cl.f, Cl.f_next = Cl.f_next, Cl.f
        Cl.m, Cl.m_next = Cl.m_next, Cl.m
        self.first_step = False
        self.time += self.hc.coarse.dt
        self.istep += 1
        if record_force and self.ib is not None:
            if pipelined:
                self._record_async(buf)
            else:
                self.flush_records()
                self.compute_ib_force()

    def step(self, n: int = 1, record_force: bool = False, pipelined: bool = False):
        if n >= 2 and not record_force and self._graph_ok():
            g = self._two_steps()
            if g is not None:
                dt = self.hc.coarse.dt
                while n >= 2:
                    capi.check(self.L.ilbm_graph_launch(self.ctx.h, g), "graph_launch")
                    self.time += 2 * dt
                    self.istep += 2
                    n -= 2
        for _ in range(n):
            self.advance(record_force=record_force, pipelined=pipelined)
        self.flush_records()

    def _graph_ok(self) -> bool:
        return (self.use_graphs and not self._graph_failed and not self.first_step and
                (self.ib_case is None or self.ib_case.geometry_type != 2))

    def _two_steps(self):
        """The graph of two coarse steps from the current buffers (which two
        steps bring back to their places), recorded once; None if recording
        fails (the steps are then taken one call at a time)."""
        if self._graph is not None:
            return self._graph
        time0, istep0 = self.time, self.istep
        capi.check(self.L.ilbm_graph_begin(self.ctx.h), "graph_begin")
        g = C.c_void_p()
        try:
            for _ in range(2):
                self._launch_step()
                Cl = self.C
                Cl.f, Cl.f_next = Cl.f_next, Cl.f
                Cl.m, Cl.m_next = Cl.m_next, Cl.m
        except Exception:
            self.L.ilbm_graph_end(self.ctx.h, C.byref(g))
            if g.value:
                self.L.ilbm_graph_destroy(g)
            # a call that cannot be recorded: the steps go one call at a
            # time (which reports a genuine error of the call itself)
            self._graph_failed = True
            return None
        finally:
            self.time, self.istep = time0, istep0
        if self.L.ilbm_graph_end(self.ctx.h, C.byref(g)) != 0 or not g.value:
            self._graph_failed = True
            return None
        self._graph = g
        return g

    def _records_with_step(self) -> bool:
        return False

    def _next_rec_buf(self):
        if self._rec_bufs is None:
            self._rec_bufs = [torch.empty(8, dtype=torch.float64, pin_memory=True) for _ in range(2)]
            self._stream = torch.cuda.ExternalStream(self.L.ilbm_stream(self.ctx.h), device=self.dev)
        buf = self._rec_bufs[self._rec_slot]
        self._rec_slot ^= 1
        return buf

    def _record_async(self, buf=None):
        """The step's record into pinned memory (buf: already taken with the
        step), its event on the library stream; the previous one is taken."""
        if buf is None:
            buf = self._next_rec_buf()
            lo, hi = self.force_region
            b = self.F.box(self.F.f, None, force=self.F.fb)
            capi.check(self.L.ilbm_force_record_async(self.ctx.h, C.byref(b), 1, self.ib, capi.ivec3(lo),
                                                      capi.ivec3(hi), buf.data_ptr()),
                       "force_record_async")
        ev = torch.cuda.Event()
        ev.record(self._stream)
        prev, self._pending = self._pending, (buf, ev)
        if prev is not None:
            self._take_record(*prev)

    def flush_records(self):
        """Takes the force record still in flight (pipelined steps)."""
        if self._pending is not None:
            prev, self._pending = self._pending, None
            self._take_record(*prev)

    _STATUS = ((0, 1, "IB stencil left the support band (marker outside its envelope)"),
               (0, 2, "IVC operator exceeded its nonzero capacity"),
               (0, 4, "IVC conjugate gradient did not converge"),
               (1, 8, "IVC operator has a non-positive pivot (not positive definite)"))

    def _take_record(self, buf, ev):
        ev.synchronize()
        r = buf.numpy().copy()
        words = (int(r[6]), int(r[7]))
        for w, bit, msg in self._STATUS:
            if words[w] & bit:
                raise capi.IlbmError(f"force_record_async: {msg}")
        self.rec = LevelSolver.force_record(self, r[0:3], r[3:6])

    def compute_ib_force(self):
        """ComputeIBForce on the finest level (AmrCoreLBM.cpp:456-631) with
        the force of the last fine substep."""
        lo, hi = self.force_region
        b = self.F.box(self.F.f, None, force=self.F.fb)
        s = (C.c_double * 3)()
        capi.check(self.L.ilbm_force_integrals(self.ctx.h, C.byref(b), 1, capi.ivec3(lo),
                                               capi.ivec3(hi), s), "force_integrals")
        m = (C.c_double * 3)()
        capi.check(self.L.ilbm_ib_last_marker_force_sum(self.ib, m), "marker_force_sum")
        self.rec = LevelSolver.force_record(self, np.array([s[0], s[1], s[2]]),
                                            np.array([m[0], m[1], m[2]]))
        return self.rec

    # ---- read-back ---------------------------------------------------------
    def _lvl(self, lev):
        return self.levels[lev]

    def get_f(self, lev: int) -> np.ndarray:
        self.ctx.sync()
        lvl = self._lvl(lev)
        v = lvl.valid(lvl.f, lvl.gf).to(torch.float64)
        if self.storage != "f64":
            w = torch.tensor(self.hc.coarse.lattice.w, dtype=torch.float64, device=self.dev).view(-1, 1, 1, 1)
            if self.storage == "f16":
                v = v * (w / self.pc.f16_scale)
            v = v + w
        return v.cpu().numpy()

    def get_macro(self, lev: int) -> np.ndarray:
        """rho, u, v, w of a level (valid cells): those of its populations
        (calculateMacroForcing with the force of its last step), and on the
        coarse cells under the fine box the averaged-down values."""
        self.ctx.sync()
        lvl = self._lvl(lev)
        if self.first_step:
            return lvl.valid(lvl.m, lvl.gm).to(torch.float64).cpu().numpy()
        out = torch.zeros_like(lvl.m)
        b = lvl.box(lvl.f, None)
        top = self.nlev - 1
        force = self.F.fb if (lev == top and self.ib is not None) else None
        p = self.params[lev]
        capi.check(self.L.ilbm_compute_macro(self.ctx.h, C.byref(b), C.byref(p), lvl.f.data_ptr(),
                                             force.data_ptr() if force is not None else None,
                                             out.data_ptr(), None, None), "compute_macro")
        self.ctx.sync()
        m = lvl.valid(out, lvl.gm).to(torch.float64).cpu().numpy()
        if lev < top:
            # the covered cells hold the averaged-down values (stored macro)
            st = lvl.valid(lvl.m, lvl.gm).to(torch.float64).cpu().numpy()
            blo, _ = self.hc.box_lohi(lev)
            flo, fhi = self.hc.box_lohi(lev + 1)
            lo = [flo[a] // 2 - blo[a] for a in range(3)]
            hi = [fhi[a] // 2 + 1 - blo[a] for a in range(3)]
            if self.dim == 3:
                sl = (slice(None), slice(lo[2], hi[2]), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
            else:
                sl = (slice(None), slice(None), slice(lo[1], hi[1]), slice(lo[0], hi[0]))
            m[sl] = st[sl]
        return m

    def get_force(self) -> np.ndarray:
        self.ctx.sync()
        return self.F.valid(self.F.fb, self.F.gm).to(torch.float64).cpu().numpy()

    def marker_force_sum(self) -> np.ndarray:
        m = (C.c_double * 3)()
        capi.check(self.L.ilbm_ib_last_marker_force_sum(self.ib, m), "marker_force_sum")
        return np.array([m[0], m[1], m[2]])

    def close(self):
        if self._graph is not None:
            self.L.ilbm_graph_destroy(self._graph)
            self._graph = None
        if self.ib is not None:
            self.L.ilbm_ib_destroy(self.ib)
            self.ib = None
        self.ctx.close()


class TwoLevelSolver(HierarchySolver):
    """A coarse level + one fine box (ratio 2) stepped by
    ``ilbm_advance_two_level``, whose schedule overlaps the coarse step with
    the fine level's body forcing."""

    def __init__(self, tl: TwoLevelCase, storage: str = "f64", ib: MarkerIB | None = None,
                 device: int = 0, f16_scale: float = 1024.0, graphs: bool = False):
        self.tl = tl
        hc = HierarchyCase(tl.coarse, ((tl.fine_lo, tl.fine_hi),), name=tl.name)
        super().__init__(hc, storage, ib, device, f16_scale, graphs)

    def set_macro(self, init_coarse, init_fine):
        super().set_macro(init_coarse, init_fine)

    def _records_with_step(self) -> bool:
        return True

    def _launch_step(self, record_into=None):
        Cl, Fl = self.C, self.F
        bc = Cl.box(Cl.f, Cl.f_next, m_in=Cl.m, m_out=Cl.m_next)
        bf = Fl.box(Fl.f, Fl.f_next, m_in=Fl.m if self.first_step else None,
                    force=Fl.fa, force_prev=Fl.fb)
        flags = capi.TWO_LEVEL_FIRST_STEP if self.first_step else 0
        if record_into is not None:  # the step and its force record (ilbm_advance_two_level_recorded)
            lo, hi = self.force_region
            capi.check(self.L.ilbm_advance_two_level_recorded(
                self.ctx.h, C.byref(bc), C.byref(self.pc), C.byref(bf), C.byref(self.pf), self.ib,
                self.tl.coarse.dt, self.time, flags, capi.ivec3(lo), capi.ivec3(hi),
                record_into.data_ptr()), "advance_two_level_recorded")
            return
        capi.check(self.L.ilbm_advance_two_level(self.ctx.h, C.byref(bc), C.byref(self.pc),
                                                 C.byref(bf), C.byref(self.pf), self.ib,
                                                 self.tl.coarse.dt, self.time, flags),
                   "advance_two_level")
