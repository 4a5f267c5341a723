"""Single-level driver over the C ABI: the host-side mirror of the reference's
per-level loop.

``LevelSolver.advance_phi_at_level()`` plays the role of
``AmrCoreLBM::AdvancePhiAtLevel`` (Source/Core/AdvanceLBMAtLevel.cpp:20-394)
for one level held in one box: optional ``IBMarkerDF::update_forcing`` on the
level, then the fused collide-stream.  ``compute_ib_force()`` mirrors
``AmrCoreLBM::ComputeIBForce`` (Source/Core/AmrCoreLBM.cpp:456-631) without the
``force.dat`` file.  Device memory comes from PyTorch (plumbing only); every
computation is a call into ``libilbm_b200.so``.

State kept between steps (the reference's f_new / macro_new / forcing):
  * ``f``      -- f^n, pre-collision populations (storage form);
  * ``force``  -- F^{n-1}, the Guo force of the last step (IB band only);
  * the macro fields are not stored: rho^n, u^n are recovered from f^n and
    F^{n-1} inside the kernels, which reproduces the stored values bit for bit
    (the reference computes them from the same data).  Step 0 reads the
    initial macro fields instead.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import capi
from .cases import LevelCase, MarkerIB

_TORCH_DT = {"f64": torch.float64, "f32": torch.float32, "f16": torch.float16}
_REAL_DT = {"f64": torch.float64, "f32": torch.float32, "f16": torch.float32}


def alloc_populations(q: int, gz: int, gy: int, gx: int, dtype, device, ngrow: int = 1) -> torch.Tensor:
    """Population array of a grown box, indexed [q, k, j, i], stored
    row-interleaved: the Q rows of one (j, k) lie next to each other, each
    row padded to a whole number of 32-byte sectors and the array shifted so
    that the first valid cell of every row (ngrow cells in) starts a sector.
    With gp the padded row length, element (i, j, k, q) of the grown box sits
    at i + gp*q + gp*Q*j + gp*Q*gy*k: an Array4 layout with component stride
    gp, j stride Q*gp and k stride Q*gp*gy, which every kernel reads through
    the strides it is given.  A level step touches the Q rows of one (j, k)
    together; keeping them within a few kilobytes of each other (instead of
    one plane apart, as AMReX's FArrayBox does) and each warp's 32 cells on
    whole sectors raised the D3Q19 FP32 level step on the 256 x 128 x 128
    sphere level from 0.677 to 0.777 of the measured HBM copy bandwidth on a
    B200, with identical results."""
    esz = torch.empty((), dtype=dtype).element_size()
    per = max(1, 32 // esz)                      # elements per 32-byte sector
    gp = (gx + per - 1) // per * per
    off = (per - ngrow % per) % per              # first valid cell on a sector
    flat = torch.zeros(gz * gy * q * gp + off, dtype=dtype, device=device)
    return flat.as_strided((q, gz, gy, gx), (gp, gy * q * gp, q * gp, 1), off)


def lattice_struct(lat) -> capi.Lattice_t:
    s = capi.Lattice_t()
    s.dim, s.q = lat.dim, lat.q
    for q in range(lat.q):
        s.cx[q], s.cy[q], s.cz[q] = lat.c[q]
        s.wis[q], s.wim[q] = lat.wis[q], lat.wim[q]
    return s


def level_params(case: LevelCase, uniform_force: bool, f16_scale: float = 1024.0) -> capi.LevelParams_t:
    p = capi.LevelParams_t()
    p.tau = case.tau
    for d in range(3):
        p.domain_lo[d] = 0
        p.domain_hi[d] = case.n_cell[d] - 1 if d < case.dim else 0
        p.periodic[d] = int(case.periodic[d]) if d < case.dim else 0
        allp = all(case.periodic[: case.dim])
        p.bc_lo[d] = case.bc_lo[d] if not allp else 0
        p.bc_hi[d] = case.bc_hi[d] if not allp else 0
        for c in range(4):
            p.bc_val_lo[d][c] = case.bc_lo_val[d][c] if not allp else 0.0
            p.bc_val_hi[d][c] = case.bc_hi_val[d][c] if not allp else 0.0
        p.force_lo[d] = 0
        p.force_hi[d] = -1
    p.ghost_mode = capi.GHOST_SELF
    if uniform_force and case.prescribed_force is not None:
        p.use_uniform_force = 1
        for d in range(3):
            p.uniform_force[d] = case.prescribed_force[d]
    p.f16_scale = f16_scale
    return p


def level_geom(case: LevelCase) -> capi.LevelGeom_t:
    g = capi.LevelGeom_t()
    g.dim = case.dim
    allp = all(case.periodic[: case.dim])
    for d in range(3):
        g.n_cell[d] = case.n_cell[d]
        g.prob_lo[d] = case.prob_lo[d]
        g.prob_hi[d] = case.prob_hi[d]
        g.periodic[d] = int(case.periodic[d]) if d < case.dim else 0
        g.bc_lo[d] = case.bc_lo[d] if not allp else 0
        g.bc_hi[d] = case.bc_hi[d] if not allp else 0
        for c in range(4):
            g.bc_val_lo[d][c] = case.bc_lo_val[d][c] if not allp else 0.0
            g.bc_val_hi[d][c] = case.bc_hi_val[d][c] if not allp else 0.0
    return g


def ib_params(ib: MarkerIB, dim: int) -> capi.IBParams_t:
    s = capi.IBParams_t()
    for name, _ in capi.IBParams_t._fields_:
        if hasattr(ib, name):
            setattr(s, name, getattr(ib, name))
    af = ib.airfoil if ib.airfoil is not None else MarkerIB.AIRFOIL_DEFAULT
    (s.airfoil_chord, s.airfoil_thickness, s.pitch_mean, s.pitch_amplitude,
     s.pitch_frequency, s.pitch_phase, s.pivot_x) = af
    if dim == 2:
        s.z0 = 0.0
    return s


class Context:
    """Owns an ``ilbm_ctx`` (lattice + storage form + stream)."""

    def __init__(self, lattice, storage: str = "f64", device: int = 0):
        self.L = capi.lib()
        self.storage = storage
        self._lat = lattice_struct(lattice)
        h = C.c_void_p()
        capi.check(self.L.ilbm_create(C.byref(self._lat), capi.STORAGE[storage], device, None,
                                      C.byref(h)), "ilbm_create")
        self.h = h

    def sync(self):
        capi.check(self.L.ilbm_sync(self.h), "ilbm_sync")

    def launches(self) -> int:
        return int(self.L.ilbm_kernel_launches(self.h))

    def record(self, slot: int):
        capi.check(self.L.ilbm_event_record(self.h, slot), "event_record")

    def elapsed_ms(self, a: int, b: int) -> float:
        ms = C.c_float()
        capi.check(self.L.ilbm_event_elapsed_ms(self.h, a, b, C.byref(ms)), "event_elapsed")
        return float(ms.value)

    def close(self):
        if getattr(self, "h", None):
            self.L.ilbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def refinement_region(case: LevelCase, ib: MarkerIB):
    """The body refinement box of ErrorEst in physical coordinates, or None
    (immersed_boundary_refinement_region, Source/Core/AmrCoreLBM.cpp:56-100;
    the pitching-airfoil hook, Examples/Pitching_airfoil/
    IBMUserDefinedGeometry.H:25-57, with the leading edge moved by pivot_x)."""
    dx = case.dx
    pad = max(6.0 * dx, 2.0)
    if ib.geometry_type == 1:
        lo = (ib.box_xlo - pad, (ib.box_yhi - pad) if ib.box_lid_only > 0 else (ib.box_ylo - pad),
              ib.box_zlo - pad)
        hi = (ib.box_xhi + pad, ib.box_yhi + pad, ib.box_zhi + pad)
        return lo, hi
    if ib.geometry_type == 2:
        if case.dim != 2:
            return None
        af = ib.airfoil if ib.airfoil is not None else MarkerIB.AIRFOIL_DEFAULT
        chord = max(af[0], 1.0e-12)
        half_t = 0.5 * af[1] * chord
        y_ext = chord * math.sin(abs(af[3])) + half_t
        le = ib.x0 - af[6]
        return (le - pad, ib.y0 - y_ext - pad, ib.z0 - pad), (le + chord + pad, ib.y0 + y_ext + pad, ib.z0 + pad)
    R = ib.R
    if R <= 0.0:
        return None
    if ib.refine_upstream > 0 and ib.refine_downstream > 0 and ib.refine_cross > 0:
        return ((ib.x0 - ib.refine_upstream * R - pad, ib.y0 - ib.refine_cross * R - pad,
                 ib.z0 - ib.refine_cross * R - pad),
                (ib.x0 + ib.refine_downstream * R + pad, ib.y0 + ib.refine_cross * R + pad,
                 ib.z0 + ib.refine_cross * R + pad))
    return ((ib.x0 - R - pad, ib.y0 - R - pad, ib.z0 - R - pad),
            (ib.x0 + R + pad, ib.y0 + R + pad, ib.z0 + R + pad))


def ib_footprint(case: LevelCase, ib: MarkerIB) -> int:
    """Estimated device bytes of an IB object: band arrays (10 doubles per
    cell of the support band), marker arrays and the IVC operator (stored
    inverse for fixed bodies up to 8192 markers, else CSR + CG vectors)."""
    d = case.dim
    ext = 2.0 * ib.R + 16.0
    if ib.geometry_type == 2 and ib.airfoil is not None:
        ext = ib.airfoil[0] + 16.0
    nb = int(ext ** d)
    h = case.dx
    area = (2.0 * math.pi * ib.R) if d == 2 else (4.0 * math.pi * ib.R * ib.R)
    n = int(max(ib.n_marker, area / (h ** (d - 1)) if ib.geometry_type == 0 else 4.0 * ext / h))
    ld = (n + 31) // 32 * 32
    op = n * ld * 8 if (ib.coupling_method == 1 and ib.geometry_type != 2 and n <= 8192) else 0
    op += n * (512 if d == 3 else 96) * 12 + n * 15 * 8 * 3
    return int(nb * 10 * 8 + n * 15 * 8 + op)


class LevelSolver:
    """One level held in one box, stepped on the GPU through the C ABI."""

    def __init__(self, case: LevelCase, storage: str = "f64", ib: MarkerIB | None = None,
                 device: int = 0, f16_scale: float = 1024.0, ctx: Context | None = None):
        if not torch.cuda.is_available():
            raise capi.IlbmError("LevelSolver needs a CUDA device")
        self.case = case
        self.storage = storage
        self.dev = torch.device("cuda", device)
        self._own_ctx = ctx is None
        self.ctx = ctx or Context(case.lattice, storage, device)
        self.L = self.ctx.L
        self.q = case.lattice.q
        self.dim = case.dim
        self.gf, self.gm = 1, 2
        nx, ny, nz = case.n_cell
        gz_f = nz + 2 * self.gf if self.dim == 3 else 1
        gz_m = nz + 2 * self.gm if self.dim == 3 else 1
        self.fshape = (self.q, gz_f, ny + 2 * self.gf, nx + 2 * self.gf)
        self.mshape_g = (gz_m, ny + 2 * self.gm, nx + 2 * self.gm)
        fdt, rdt = _TORCH_DT[storage], _REAL_DT[storage]
        self.f = alloc_populations(*self.fshape, fdt, self.dev, ngrow=self.gf)
        self.f_next = alloc_populations(*self.fshape, fdt, self.dev, ngrow=self.gf)
        self.macro = torch.zeros((4,) + self.mshape_g, dtype=rdt, device=self.dev)
        self.force_cur = torch.zeros((3,) + self.mshape_g, dtype=rdt, device=self.dev)
        self.force_prev = torch.zeros((3,) + self.mshape_g, dtype=rdt, device=self.dev)
        self.f16_scale = f16_scale
        self.params = level_params(case, uniform_force=(ib is None), f16_scale=f16_scale)
        self.ib = None
        self.ib_case = ib
        if ib is not None:
            self._geom = level_geom(case)
            self._ibp = ib_params(ib, self.dim)
            h = C.c_void_p()
            capi.check(self.L.ilbm_ib_create(self.ctx.h, C.byref(self._ibp), C.byref(self._geom),
                                             C.byref(h)), "ilbm_ib_create")
            self.ib = h
            lo, hi = (C.c_int * 3)(), (C.c_int * 3)()
            capi.check(self.L.ilbm_ib_force_region(self.ib, lo, hi), "ib_force_region")
            for d in range(3):
                self.params.force_lo[d], self.params.force_hi[d] = lo[d], hi[d]
            self.force_region = (tuple(lo), tuple(hi))
        self.time = 0.0
        self.istep = 0
        self.first_step_macro = False
        self.have_prev_body = False
        self.prev_body = np.zeros(3)
        self.rec = np.zeros(18)
        self.ib_ready = False  # the body's IVC operator is built by its first step

    # ---- layout helpers ---------------------------------------------------
    def _box(self, f_in, f_out, macro_in=None, macro_out=None, force=None, force_prev=None):
        b = capi.Box_t()
        for d in range(3):
            b.lo[d] = 0
            b.hi[d] = self.case.n_cell[d] - 1 if d < self.dim else 0
        b.ngrow_f, b.ngrow_m = self.gf, self.gm
        fs = self.f.stride()
        b.fstride[0], b.fstride[1], b.fstride[2] = fs[2], fs[1], fs[0]
        ms = self.macro.stride()
        b.mstride[0], b.mstride[1], b.mstride[2] = ms[2], ms[1], ms[0]
        b.f_in = f_in.data_ptr()
        b.f_out = f_out.data_ptr() if f_out is not None else None
        b.macro_in = macro_in.data_ptr() if macro_in is not None else None
        b.macro_out = macro_out.data_ptr() if macro_out is not None else None
        b.force = force.data_ptr() if force is not None else None
        b.force_prev = force_prev.data_ptr() if force_prev is not None else None
        return b

    def _valid(self, t, g):
        nx, ny, nz = self.case.n_cell
        if self.dim == 3:
            return t[..., g:g + nz, g:g + ny, g:g + nx]
        return t[..., :, g:g + ny, g:g + nx]

    # ---- initialisation (MakeNewLevelFromScratch + InitEquilibrium) --------
    def set_macro(self, rho, ux, uy, uz=None):
        """Initial macro fields on valid cells ([nz, ny, nx]); f = f_eq(rho, u)."""
        v = self._valid(self.macro, self.gm)
        rdt = self.macro.dtype
        v[0].copy_(torch.as_tensor(np.asarray(rho), dtype=rdt))
        v[1].copy_(torch.as_tensor(np.asarray(ux), dtype=rdt))
        v[2].copy_(torch.as_tensor(np.asarray(uy), dtype=rdt))
        if uz is not None:
            v[3].copy_(torch.as_tensor(np.asarray(uz), dtype=rdt))
        torch.cuda.synchronize(self.dev)
        b = self._box(self.f, self.f_next, macro_in=self.macro)
        capi.check(self.L.ilbm_init_equilibrium(self.ctx.h, C.byref(b)), "init_equilibrium")
        self.ctx.sync()
        self.first_step_macro = True
        self.time = 0.0
        self.istep = 0

    def set_f(self, f):
        """Populations f^n (unshifted, float64, [Q, nz, ny, nx]) on valid cells."""
        f = torch.as_tensor(np.asarray(f, dtype=np.float64))
        if self.storage != "f64":
            w = torch.tensor(self.case.lattice.w, dtype=torch.float64).view(-1, 1, 1, 1)
            f = f - w
            if self.storage == "f16":
                f = f * (self.f16_scale / w)
        self._valid(self.f, self.gf).copy_(f.to(self.f.dtype))
        torch.cuda.synchronize(self.dev)
        self.first_step_macro = False

    def set_force_prev(self, F):
        """F^{n-1} on valid cells ([3, nz, ny, nx]) -- the force of the step that produced f."""
        self._valid(self.force_prev, self.gm).copy_(torch.as_tensor(np.asarray(F), dtype=self.force_prev.dtype))
        torch.cuda.synchronize(self.dev)

    # ---- the level step ---------------------------------------------------
    def advance_phi_at_level(self, record_force: bool = False):
        use_macro = self.macro if self.first_step_macro else None
        ib_on = self.ib is not None
        b = self._box(self.f, self.f_next, macro_in=use_macro,
                      force=self.force_cur if ib_on else None,
                      force_prev=self.force_prev if ib_on else None)
        # update_forcing + collide-stream (the IB chain overlaps the cells
        # outside its band inside the library)
        capi.check(self.L.ilbm_advance_level(self.ctx.h, C.byref(b), C.byref(self.params),
                                             self.ib, self.case.dt, self.time), "advance_level")
        self.f, self.f_next = self.f_next, self.f
        self.force_cur, self.force_prev = self.force_prev, self.force_cur
        self.first_step_macro = False
        self.ib_ready = ib_on
        self.time += self.case.dt
        self.istep += 1
        if record_force and ib_on:
            self.compute_ib_force()

    def step(self, n: int = 1, record_force: bool = False):
        for _ in range(n):
            self.advance_phi_at_level(record_force=record_force)

    def run_recorded(self, n: int) -> np.ndarray:
        """n steps queued back to back, each followed by its force record
        copied to pinned host memory in stream order
        (ilbm_force_record_async), with one synchronisation at the end;
        returns the n force records (the rows of force_record).  Without a
        body it is n plain steps and returns an empty array."""
        if self.ib is None:
            self.step(n)
            self.ctx.sync()
            return np.zeros((0, 18))
        buf = torch.empty((n, 8), dtype=torch.float64, pin_memory=True)
        lo, hi = self.force_region
        lo3, hi3 = capi.ivec3(lo), capi.ivec3(hi)
        for i in range(n):
            self.advance_phi_at_level()
            b = self._box(self.f, None, force=self.force_prev)
            capi.check(self.L.ilbm_force_record_async(self.ctx.h, C.byref(b), 1, self.ib, lo3, hi3,
                                                      buf[i].data_ptr()), "force_record_async")
        self.ctx.sync()
        r = buf.numpy().copy()
        for w, bit, msg in ((0, 1, "IB stencil left the support band"), (0, 2, "IVC operator capacity"),
                            (0, 4, "IVC conjugate gradient did not converge"),
                            (1, 8, "IVC operator has a non-positive pivot")):
            if np.any(r[:, 6 + w].astype(np.int64) & bit):
                raise capi.IlbmError(f"force_record_async: {msg}")
        recs = self.force_records(r[:, 0:3], r[:, 3:6])
        self.rec = recs[-1].copy()
        return recs

    # ---- force evaluation (ComputeIBForce, AmrCoreLBM.cpp:456-631) --------
    def compute_ib_force(self):
        lo, hi = self.force_region
        b = self._box(self.f, None, force=self.force_prev)
        s = (C.c_double * 3)()
        capi.check(self.L.ilbm_force_integrals(self.ctx.h, C.byref(b), 1, capi.ivec3(lo),
                                               capi.ivec3(hi), s), "force_integrals")
        m = (C.c_double * 3)()
        capi.check(self.L.ilbm_ib_last_marker_force_sum(self.ib, m), "marker_force_sum")
        self.rec = self.force_record(np.array([s[0], s[1], s[2]]), np.array([m[0], m[1], m[2]]))
        return self.rec

    def force_record(self, eul_sum, marker_sum):
        """One line of the force record from the Eulerian force sum over the IB
        force region and the marker force sum of a step (ComputeIBForce,
        AmrCoreLBM.cpp:489-631): body force, time-centred with the previous
        step's, and Cd / Cl.  Layout: Ftc(3), Cd, Cl, Cz, Fb(3), Feul(3),
        Fmarker(3), Fme(3)."""
        case, ib = self.case, self.ib_case
        Fs = np.array([eul_sum[0], eul_sum[1], eul_sum[2] if self.dim == 3 else 0.0])
        dV = case.dx ** self.dim
        Feul = -(Fs * dV) / case.dt
        Fm = -np.asarray(marker_sum, dtype=np.float64)
        Fme = Feul.copy()
        Fb = {0: Fme, 1: Feul, 2: Fm}.get(ib.force_eval_method, Feul)
        Ftc = 0.5 * (self.prev_body + Fb) if self.have_prev_body else Fb.copy()
        self.prev_body = Fb.copy()
        self.have_prev_body = True
        U = ib.U0
        denom = (0.5 * 1.0 * U * U * (math.pi * ib.R * ib.R)) if self.dim == 3 else (0.5 * 1.0 * U * U * (2.0 * ib.R))
        rec = np.zeros(18)
        rec[0:3], rec[6:9], rec[9:12], rec[12:15], rec[15:18] = Ftc, Fb, Feul, Fm, Fme
        if denom > 0:
            rec[3], rec[4] = Ftc[0] / denom, Ftc[1] / denom
            if self.dim == 3:
                rec[5] = Ftc[2] / denom
        return rec

    def force_records(self, eul_sums: np.ndarray, marker_sums: np.ndarray) -> np.ndarray:
        """force_record for a run of consecutive steps at once: rows of
        Eulerian and marker force sums in, rows of the 18-value record out
        (the same elementwise arithmetic, so the same values), with the
        previous-step state carried through and left at the last step."""
        case, ib = self.case, self.ib_case
        n = len(eul_sums)
        if n == 0:
            return np.zeros((0, 18))
        Fs = np.array(eul_sums, dtype=np.float64).reshape(n, 3).copy()
        if self.dim != 3:
            Fs[:, 2] = 0.0
        dV = case.dx ** self.dim
        Feul = -(Fs * dV) / case.dt
        Fm = -np.asarray(marker_sums, dtype=np.float64).reshape(n, 3)
        Fme = Feul.copy()
        Fb = {0: Fme, 1: Feul, 2: Fm}.get(ib.force_eval_method, Feul)
        prev = np.vstack([self.prev_body[None, :], Fb[:-1]])
        Ftc = 0.5 * (prev + Fb)
        if not self.have_prev_body:
            Ftc[0] = Fb[0]
        self.prev_body = Fb[-1].copy()
        self.have_prev_body = True
        U = ib.U0
        denom = (0.5 * 1.0 * U * U * (math.pi * ib.R * ib.R)) if self.dim == 3 else (0.5 * 1.0 * U * U * (2.0 * ib.R))
        rec = np.zeros((n, 18))
        rec[:, 0:3], rec[:, 6:9], rec[:, 9:12], rec[:, 12:15], rec[:, 15:18] = Ftc, Fb, Feul, Fm, Fme
        if denom > 0:
            rec[:, 3], rec[:, 4] = Ftc[:, 0] / denom, Ftc[:, 1] / denom
            if self.dim == 3:
                rec[:, 5] = Ftc[:, 2] / denom
        return rec

    # ---- read-back ---------------------------------------------------------
    def get_f(self) -> np.ndarray:
        self.ctx.sync()
        v = self._valid(self.f, self.gf).to(torch.float64)
        if self.storage != "f64":
            w = torch.tensor(self.case.lattice.w, dtype=torch.float64, device=self.dev).view(-1, 1, 1, 1)
            if self.storage == "f16":
                v = v * (w / self.f16_scale)
            v = v + w
        return v.cpu().numpy()

    def get_macro(self) -> np.ndarray:
        """rho, u, v, w of the current state (calculateMacroForcing with F^{n-1})."""
        out = torch.zeros_like(self.macro)
        b = self._box(self.f, None)
        p = self.params
        force = self.force_prev if self.ib is not None else None
        capi.check(self.L.ilbm_compute_macro(self.ctx.h, C.byref(b), C.byref(p), self.f.data_ptr(),
                                             force.data_ptr() if force is not None else None,
                                             out.data_ptr(), None, None), "compute_macro")
        self.ctx.sync()
        return self._valid(out, self.gm).to(torch.float64).cpu().numpy()

    # ---- derived fields and refinement tags (UpdateDerivedMacroFields, ErrorEst)
    def derived_fields(self):
        """(vorticity, pressure, max vorticity) of the current state on valid
        cells (device tensors kept in self.vor / self.pres)."""
        self.vor = torch.zeros_like(self.macro[0])
        self.pres = torch.zeros_like(self.macro[0])
        b = self._box(self.f, None)
        force = self.force_prev if self.ib is not None else None
        vmax = C.c_double()
        capi.check(self.L.ilbm_derived_fields(self.ctx.h, C.byref(b), C.byref(self.params),
                                              self.f.data_ptr(),
                                              force.data_ptr() if force is not None else None,
                                              capi.dvec3([self.case.dx] * 3), self.vor.data_ptr(),
                                              self.pres.data_ptr(), C.byref(vmax)), "derived_fields")
        to_np = lambda t: self._valid(t, self.gm).to(torch.float64).cpu().numpy()
        return to_np(self.vor), to_np(self.pres), vmax.value

    def tag_cells(self, threshold_ratio: float = 1.0, refine_box=True, no_refine=(0.0, 0.0),
                  levelset=True, n_cells_band: int = 5):
        """ErrorEst tags of the current state: (tags [nz, ny, nx] of 0/1,
        number tagged, threshold).  refine_box: True for the body's refinement
        region (when there is a body), a (lo, hi) pair, or False.  levelset:
        also tag the signed-distance band of a cylinder / sphere body (the
        reference's cylinder-geometry branch), when there is one."""
        _, _, vmax = self.derived_fields()
        ls = None
        if levelset and self.ib_case is not None and self.ib_case.geometry_type == 0:
            m = self.ib_case
            ls = (C.c_double * 6)(m.x0, m.y0, m.z0 if self.dim == 3 else 0.0, m.R,
                                  float(n_cells_band), self.case.dx)
        threshold = threshold_ratio * vmax
        box = None
        if refine_box is True and self.ib_case is not None:
            box = refinement_region(self.case, self.ib_case)
        elif refine_box not in (True, False, None):
            box = refine_box
        nx, ny, nz = self.case.n_cell
        tags = torch.zeros(nx * ny * (nz if self.dim == 3 else 1), dtype=torch.uint8, device=self.dev)
        b = self._box(self.f, None)
        cnt = C.c_int64()
        capi.check(self.L.ilbm_tag_cells(self.ctx.h, C.byref(b), self.vor.data_ptr(), threshold,
                                         int(box is not None),
                                         capi.dvec3(box[0]) if box is not None else None,
                                         capi.dvec3(box[1]) if box is not None else None,
                                         float(no_refine[0]), float(no_refine[1]),
                                         capi.dvec3(self.case.prob_lo), capi.dvec3(self.case.prob_hi),
                                         capi.dvec3([self.case.dx] * 3), ls, tags.data_ptr(),
                                         C.byref(cnt)), "tag_cells")
        shape = (nz, ny, nx) if self.dim == 3 else (1, ny, nx)
        return tags.cpu().numpy().reshape(shape), cnt.value, threshold

    # ---- state I/O (checkpoint / restart, plotfile) ------------------------
    def save_checkpoint(self, path) -> None:
        """Checkpoint of the level: f^n, F^{n-1} and the body when there is one,
        the stored macro fields when the next step still reads them, and this
        object's step count, time and force-record history (the
        WriteCheckpointFile the reference leaves as a stub,
        Source/Core/AmrCoreLBM.cpp:1932-2010)."""
        b = self._box(self.f, None, macro_in=self.macro if self.first_step_macro else None,
                      force_prev=self.force_prev if self.ib is not None else None)
        m = capi.CheckpointMeta_t()
        m.istep, m.time = self.istep, self.time
        m.user[0] = 1.0 if self.have_prev_body else 0.0
        m.user[1], m.user[2], m.user[3] = (float(v) for v in self.prev_body)
        capi.check(self.L.ilbm_checkpoint_write(self.ctx.h, C.byref(b), self.ib, C.byref(m),
                                                str(path).encode()), "checkpoint_write")

    def load_checkpoint(self, path) -> None:
        """Restores a checkpoint written by save_checkpoint on a solver made
        with the same case, storage and body; the next step continues the saved
        run bit for bit (ReadCheckpointFile, AmrCoreLBM.cpp:2020-2115)."""
        b = self._box(self.f, None, macro_in=self.macro,
                      force_prev=self.force_prev if self.ib is not None else None)
        m = capi.CheckpointMeta_t()
        capi.check(self.L.ilbm_checkpoint_read(self.ctx.h, C.byref(b), self.ib, C.byref(m),
                                               str(path).encode()), "checkpoint_read")
        self.istep, self.time = int(m.istep), float(m.time)
        self.first_step_macro = bool(m.flags & capi.CKPT_MACRO)
        self.have_prev_body = m.user[0] != 0.0
        self.prev_body = np.array([m.user[1], m.user[2], m.user[3]])
        self.ib_ready = False

    def write_plotfile(self, path, levelset: bool | None = None) -> None:
        """AMReX plotfile of the current state (WritePlotFile,
        AmrCoreLBM.cpp:1908-1930): rho, ux, uy, uz, vor, Pressure,
        f_new_0..Q-1 and, for a cylinder / sphere body (levelset None picks
        that), phi with the body's interior masked as PlotFileMF does."""
        if levelset is None:
            levelset = self.ib_case is not None and self.ib_case.geometry_type == 0
        b = self._box(self.f, None, force_prev=self.force_prev if self.ib is not None else None)
        c = self.case
        info = capi.PlotInfo_t()
        for d in range(3):
            info.prob_lo[d], info.prob_hi[d], info.dx[d] = c.prob_lo[d], c.prob_hi[d], c.dx
        info.time, info.istep = self.time, self.istep
        if levelset:
            m = self.ib_case
            info.levelset = 1
            info.ls_center[0], info.ls_center[1], info.ls_center[2] = m.x0, m.y0, m.z0
            info.ls_radius = m.R
            info.body_u[0], info.body_u[1], info.body_u[2] = m.ubx, m.uby, m.ubz
        capi.check(self.L.ilbm_plotfile_write(self.ctx.h, C.byref(b), C.byref(self.params),
                                              C.byref(info), str(path).encode()), "plotfile_write")

    def mean_velocity(self) -> np.ndarray:
        """Domain-mean velocity of the current state (reduced on the device)."""
        out = torch.zeros_like(self.macro)
        b = self._box(self.f, None)
        force = self.force_prev if self.ib is not None else None
        capi.check(self.L.ilbm_compute_macro(self.ctx.h, C.byref(b), C.byref(self.params),
                                             self.f.data_ptr(),
                                             force.data_ptr() if force is not None else None,
                                             out.data_ptr(), None, None), "compute_macro")
        self.ctx.sync()
        v = self._valid(out, self.gm)[1:4].to(torch.float64)
        return v.reshape(3, -1).mean(dim=1).cpu().numpy()

    def footprint_bytes(self) -> int:
        """Device memory this solver holds (fields; IB arrays estimated)."""
        n = sum(t.untyped_storage().nbytes()
                for t in (self.f, self.f_next, self.macro, self.force_cur, self.force_prev))
        if self.ib is not None:
            n += ib_footprint(self.case, self.ib_case)
        return int(n)

    def get_force(self) -> np.ndarray:
        """Force F used in the last step ([3, nz, ny, nx])."""
        self.ctx.sync()
        if self.ib is None:
            sh = (3,) + self.case.shape
            pf = self.case.prescribed_force or (0.0, 0.0, 0.0)
            return np.stack([np.full(self.case.shape, pf[d]) for d in range(3)]).reshape(sh)
        return self._valid(self.force_prev, self.gm).to(torch.float64).cpu().numpy()

    def num_markers(self) -> int:
        n = C.c_int64()
        capi.check(self.L.ilbm_ib_num_markers(self.ib, C.byref(n)), "num_markers")
        return int(n.value)

    def marker_force_sum(self) -> np.ndarray:
        m = (C.c_double * 3)()
        capi.check(self.L.ilbm_ib_last_marker_force_sum(self.ib, m), "marker_force_sum")
        return np.array([m[0], m[1], m[2]])

    def set_ivc_solver(self, solver: int):
        """capi.IVC_AUTO / IVC_CG / IVC_DENSE (see ilbm_ib_set_ivc_solver)."""
        capi.check(self.L.ilbm_ib_set_ivc_solver(self.ib, int(solver)), "ib_set_ivc_solver")

    def cg_iterations(self) -> int:
        it = C.c_int()
        capi.check(self.L.ilbm_ib_solver_stats(self.ib, C.byref(it)), "ib_solver_stats")
        return int(it.value)

    def markers(self):
        n = self.num_markers()
        xyz, uvw, F = (np.zeros(3 * n) for _ in range(3))
        dp = C.POINTER(C.c_double)
        capi.check(self.L.ilbm_ib_markers(self.ib, xyz.ctypes.data_as(dp), uvw.ctypes.data_as(dp),
                                          F.ctypes.data_as(dp)), "ib_markers")
        return xyz.reshape(3, n).T, uvw.reshape(3, n).T, F.reshape(3, n).T

    def momentum_exchange(self, x0, y0, z0, R, one_sided=False) -> np.ndarray:
        b = self._box(self.f, None)
        out = (C.c_double * 3)()
        dx = [self.case.dx] * 3
        capi.check(self.L.ilbm_momentum_exchange(self.ctx.h, C.byref(b), 1, C.byref(self.params),
                                                 x0, y0, z0, R,
                                                 capi.dvec3(self.case.prob_lo), capi.dvec3(dx),
                                                 int(one_sided), out), "momentum_exchange")
        return np.array([out[0], out[1], out[2]])

    def close(self):
        if self.ib is not None:
            self.L.ilbm_ib_destroy(self.ib)
            self.ib = None
        if self.ctx is not None and self._own_ctx:
            self.ctx.close()
        self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
