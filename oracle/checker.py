"""ctypes access to the CPU checkers: TEST INFRASTRUCTURE ONLY.

Two interchangeable backends with the same API:

* ``"oracle"`` -- ``_ref/liblbm_oracle.so``: the plain-C FP64 restatement in
  ``lbm_oracle.c``;
* ``"ref"``    -- ``_ref/libref{2,3}d_f{64,32}.so``: the reference's own
  sources compiled in place against ``amrex_shim/`` (see ``ref_driver.cpp``).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only to check or to time the CPU path.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF_DIR = HERE / "_ref"
MAXQ = 27
FORCE_REC = 18


class IlbmCase(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("q", C.c_int),
        ("cx", C.c_double * MAXQ), ("cy", C.c_double * MAXQ), ("cz", C.c_double * MAXQ),
        ("wis", C.c_double * MAXQ), ("wim", C.c_double * MAXQ),
        ("n_cell", C.c_int * 3),
        ("prob_lo", C.c_double * 3), ("prob_hi", C.c_double * 3),
        ("periodic", C.c_int * 3),
        ("bc_lo", C.c_int * 3), ("bc_hi", C.c_int * 3),
        ("bc_lo_rho", C.c_double * 3), ("bc_lo_ux", C.c_double * 3),
        ("bc_lo_uy", C.c_double * 3), ("bc_lo_uz", C.c_double * 3),
        ("bc_hi_rho", C.c_double * 3), ("bc_hi_ux", C.c_double * 3),
        ("bc_hi_uy", C.c_double * 3), ("bc_hi_uz", C.c_double * 3),
        ("nu", C.c_double),
        ("use_prescribed_force", C.c_int),
        ("prescribed_force", C.c_double * 3),
        ("nghost", C.c_int),
    ]


class IlbmIbCase(C.Structure):
    _fields_ = [
        ("coupling_method", C.c_int), ("delta_type", C.c_int), ("loop_ns", C.c_int),
        ("mdf_relax", C.c_double), ("explicit_diag_eps", C.c_double),
        ("geometry_type", C.c_int),
        ("box_xlo", C.c_double), ("box_xhi", C.c_double), ("box_ylo", C.c_double),
        ("box_yhi", C.c_double), ("box_zlo", C.c_double), ("box_zhi", C.c_double),
        ("box_ds", C.c_double),
        ("box_lid_only", C.c_int),
        ("box_lid_ux", C.c_double), ("box_lid_uy", C.c_double), ("box_lid_uz", C.c_double),
        ("box_wall_tol", C.c_double),
        ("n_marker", C.c_int),
        ("rd", C.c_double),
        ("ubx", C.c_double), ("uby", C.c_double), ("ubz", C.c_double),
        ("omx", C.c_double), ("omy", C.c_double), ("omz", C.c_double),
        ("ivc_diag_reg", C.c_double),
        ("ivc_rebuild_matrix", C.c_int),
        ("renormalize_delta", C.c_int),
        ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("R", C.c_double),
        ("force_eval_method", C.c_int),
        ("U0", C.c_double),
    ]


def to_case(spec) -> IlbmCase:
    """Build the checker's case struct from an ``ilbmrex_b200.cases.LevelCase``."""
    c = IlbmCase()
    lat = spec.lattice
    c.dim, c.q = lat.dim, lat.q
    for q in range(lat.q):
        c.cx[q], c.cy[q], c.cz[q] = lat.c[q]
        c.wis[q], c.wim[q] = lat.wis[q], lat.wim[q]
    for d in range(3):
        c.n_cell[d] = spec.n_cell[d]
        c.prob_lo[d] = spec.prob_lo[d]
        c.prob_hi[d] = spec.prob_hi[d]
        c.periodic[d] = int(spec.periodic[d])
        c.bc_lo[d], c.bc_hi[d] = spec.bc_lo[d], spec.bc_hi[d]
        c.bc_lo_rho[d], c.bc_lo_ux[d], c.bc_lo_uy[d], c.bc_lo_uz[d] = spec.bc_lo_val[d]
        c.bc_hi_rho[d], c.bc_hi_ux[d], c.bc_hi_uy[d], c.bc_hi_uz[d] = spec.bc_hi_val[d]
    c.nu = spec.nu
    c.use_prescribed_force = int(spec.prescribed_force is not None)
    if spec.prescribed_force is not None:
        for d in range(3):
            c.prescribed_force[d] = spec.prescribed_force[d]
    c.nghost = spec.nghost
    return c


def to_ib_case(ib) -> IlbmIbCase:
    """Build the checker's IB struct from an ``ilbmrex_b200.cases.MarkerIB``."""
    s = IlbmIbCase()
    for name, _ in IlbmIbCase._fields_:
        setattr(s, name, getattr(ib, name))
    return s


def _lib(path: Path, prefix: str):
    lib = C.CDLL(str(path))
    P, I, D, L = C.c_void_p, C.c_int, C.c_double, C.c_long
    dp = C.POINTER(C.c_double)
    sig = {
        "create": (P, [C.POINTER(IlbmCase)]),
        "destroy": (None, [P]),
        "set_macro": (I, [P, dp]),
        "init_equilibrium": (I, [P]),
        "set_f": (I, [P, dp]),
        "get_f": (I, [P, dp]),
        "get_macro": (I, [P, dp]),
        "get_force": (I, [P, dp]),
        "set_forcing": (I, [P, dp]),
        "ib_create": (I, [P, C.POINTER(IlbmIbCase)]),
        "ib_num_markers": (L, [P]),
        "ib_marker_force_sum": (I, [P, dp]),
        "step": (I, [P, I]),
        "time": (D, [P]),
        "tau": (D, [P]),
        "force_record": (I, [P, dp]),
        "momentum_exchange": (I, [P, D, D, D, D, I, dp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, prefix + name)
        fn.restype, fn.argtypes = res, args
    return lib


_LIBS: dict = {}


def _load(backend: str, dim: int, fp32: bool = False):
    key = (backend, dim, fp32)
    if key not in _LIBS:
        if backend == "oracle":
            path = REF_DIR / "liblbm_oracle.so"
            lib = _lib(path, "orc_")
            for name, res, args in [
                ("orc_fill_patch_f", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
                ("orc_fill_patch_macro", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
                ("orc_grown_cells", C.c_long, [C.c_void_p]),
                ("orc_ib_dv", C.c_double, [C.c_void_p]),
                ("orc_ib_marker_state", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
                ("orc_ib_marker_force", C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
                ("orc_set_airfoil", None, [C.POINTER(C.c_double)]),
                ("orc_delta_function", C.c_double, [C.c_double] * 3 + [C.c_int]),
                ("orc_overlap", C.c_double, [C.c_double] * 3 + [C.c_int, C.c_double, C.c_int, C.c_int]),
                ("orc_set_spread_order", None, [C.c_int]),
            ]:
                fn = getattr(lib, name)
                fn.restype, fn.argtypes = res, args
        else:
            path = REF_DIR / f"libref{dim}d_f{'32' if fp32 else '64'}.so"
            lib = _lib(path, "ref_")
            for name, res, args in [
                ("ref_set_threads", C.c_int, [C.c_int]),
                ("ref_ib_marker_state", C.c_int, [C.c_void_p, C.c_double, C.POINTER(C.c_double), C.c_long]),
                ("ref_delta_function", C.c_double, [C.c_double] * 3 + [C.c_int]),
                ("ref_overlap_1d", C.c_double, [C.c_double] * 3 + [C.c_int, C.c_double, C.c_int, C.c_int]),
                ("ref_feq", C.c_double, [C.c_double] * 8),
                ("ref_derived", C.c_int, [C.c_void_p] + [C.POINTER(C.c_double)] * 3),
                ("ref_tags", C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.c_double, C.c_int,
                                       C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_double,
                                       C.c_double, C.POINTER(C.c_double), C.c_char_p]),
            ]:
                fn = getattr(lib, name)
                fn.restype, fn.argtypes = res, args
        _LIBS[key] = lib
    return _LIBS[key]


def set_spread_order(reverse: bool) -> None:
    """Marker order of the oracle's force spreading for every level of the
    process: False = marker order (the reference's), True = reversed.  Used
    to measure how much the reference's result depends on the summation
    order of spreading alone."""
    for dim in (2, 3):
        _load("oracle", dim).orc_set_spread_order(1 if reverse else 0)


def available(backend: str = "oracle", dim: int = 2, fp32: bool = False) -> bool:
    if backend == "oracle":
        return (REF_DIR / "liblbm_oracle.so").exists()
    return (REF_DIR / f"libref{dim}d_f{'32' if fp32 else '64'}.so").exists()


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class CpuLevel:
    """One level held in one box, advanced by a CPU checker backend."""

    def __init__(self, spec, backend: str = "oracle", fp32: bool = False, threads: int | None = None):
        self.spec = spec
        self.backend = backend
        self.dim = spec.lattice.dim
        self.q = spec.lattice.q
        self.lib = _load(backend, self.dim, fp32)
        self.p = "orc_" if backend == "oracle" else "ref_"
        if backend == "ref" and threads is not None:
            self.lib.ref_set_threads(int(threads))
        self._case = to_case(spec)
        self.h = self._fn("create")(C.byref(self._case))
        if not self.h:
            raise RuntimeError(f"{backend}: create failed")
        self.shape = tuple(spec.shape)  # (nz, ny, nx); nz = 1 in 2D
        self.ncell = int(np.prod(self.shape))

    def _fn(self, name):
        return getattr(self.lib, self.p + name)

    def close(self):
        if self.h:
            self._fn("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{self.backend}: {what} failed ({rc})")

    def set_macro(self, rho, ux, uy, uz=None):
        m = np.zeros((4,) + self.shape)
        m[0], m[1], m[2] = rho, ux, uy
        if uz is not None:
            m[3] = uz
        m = np.ascontiguousarray(m, dtype=np.float64)
        self._chk(self._fn("set_macro")(self.h, _dp(m)), "set_macro")

    def init_equilibrium(self):
        self._chk(self._fn("init_equilibrium")(self.h), "init_equilibrium")

    def set_f(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64).reshape((self.q,) + self.shape)
        self._chk(self._fn("set_f")(self.h, _dp(f)), "set_f")

    def get_f(self):
        out = np.zeros((self.q,) + self.shape)
        self._chk(self._fn("get_f")(self.h, _dp(out)), "get_f")
        return out

    def get_macro(self):
        out = np.zeros((4,) + self.shape)
        self._chk(self._fn("get_macro")(self.h, _dp(out)), "get_macro")
        return out

    def get_force(self):
        out = np.zeros((3,) + self.shape)
        self._chk(self._fn("get_force")(self.h, _dp(out)), "get_force")
        return out

    def ib_create(self, ib):
        if self.backend == "oracle" and getattr(ib, "airfoil", None) is not None:
            p = np.ascontiguousarray(np.asarray(ib.airfoil, dtype=np.float64))
            self.lib.orc_set_airfoil(_dp(p))
        self._ib = to_ib_case(ib)
        self._chk(self._fn("ib_create")(self.h, C.byref(self._ib)), "ib_create")

    def num_markers(self) -> int:
        return int(self._fn("ib_num_markers")(self.h))

    def marker_force_sum(self):
        out = np.zeros(3)
        self._chk(self._fn("ib_marker_force_sum")(self.h, _dp(out)), "marker_force_sum")
        return out

    def step(self, n: int = 1):
        self._chk(self._fn("step")(self.h, int(n)), "step")

    @property
    def time(self) -> float:
        return float(self._fn("time")(self.h))

    @property
    def tau(self) -> float:
        return float(self._fn("tau")(self.h))

    def force_record(self):
        out = np.zeros(FORCE_REC)
        self._fn("force_record")(self.h, _dp(out))
        return out

    def momentum_exchange(self, x0, y0, z0, R, one_sided=False):
        out = np.zeros(3)
        self._chk(self._fn("momentum_exchange")(self.h, x0, y0, z0, R, int(one_sided), _dp(out)),
                  "momentum_exchange")
        return out

    # oracle-only helpers
    def fill_patch_f(self):
        n = int(self.lib.orc_grown_cells(self.h))
        out = np.zeros(self.q * n)
        self.lib.orc_fill_patch_f(self.h, _dp(out))
        return out

    def fill_patch_macro(self):
        n = int(self.lib.orc_grown_cells(self.h))
        out = np.zeros(6 * n)
        self.lib.orc_fill_patch_macro(self.h, _dp(out))
        return out

    def marker_state(self):
        n = self.num_markers()
        out = np.zeros(6 * n)
        if self.backend == "oracle":
            self.lib.orc_ib_marker_state(self.h, _dp(out))
        else:
            self.lib.ref_ib_marker_state(self.h, self.time, _dp(out), n)
        return out.reshape(n, 6)

    def ref_derived(self):
        """(vorticity, pressure, vortMax) from the reference build's visPara on
        its FillPatched macro_new (valid cells, [nz, ny, nx])."""
        vor, pres, vm = np.zeros(self.ncell), np.zeros(self.ncell), C.c_double()
        self._chk(self.lib.ref_derived(self.h, _dp(vor), _dp(pres), C.byref(vm)), "derived")
        return vor.reshape(self.shape), pres.reshape(self.shape), vm.value

    def ref_tags(self, vor, threshold, box=None, no_refine=(0.0, 0.0), levelset=None):
        """ErrorEst tags from the reference build's Tagging.H functions."""
        v = np.ascontiguousarray(vor, dtype=np.float64).reshape(-1)
        out = C.create_string_buffer(self.ncell)
        dv = lambda a: (C.c_double * len(a))(*a)
        rc = self.lib.ref_tags(self.h, _dp(v), float(threshold), int(box is not None),
                               dv(box[0]) if box is not None else None,
                               dv(box[1]) if box is not None else None,
                               float(no_refine[0]), float(no_refine[1]),
                               dv(levelset) if levelset is not None else None, out)
        self._chk(rc, "tags")
        return np.frombuffer(out.raw, dtype=np.uint8).reshape(self.shape).copy()

    def marker_dv(self) -> float:
        return float(self.lib.orc_ib_dv(self.h))


class CpuHierarchy:
    """A static hierarchy advanced by the oracle (orcN_*): coarse level = the
    domain, one box per finer level (ratio 2, properly nested), two substeps
    of each finer level per step of the level above with coarse-fine ghosts
    from that level's macro fields, average-down after them.  `hc` has
    ``coarse`` (LevelCase), ``boxes`` ((lo, hi) per finer level in its own
    domain indices), ``nlev`` and ``box_case(l)``."""

    def __init__(self, hc):
        self.hc = hc
        self.nlev = hc.nlev
        self.lib = _load("oracle", hc.coarse.dim)
        lib = self.lib
        P, I = C.c_void_p, C.c_int
        ip = C.POINTER(C.c_int)
        for name, res, args in [("orcN_create", P, [C.POINTER(IlbmCase), I, ip]),
                                ("orcN_destroy", None, [P]), ("orcN_level", P, [P, I]),
                                ("orcN_step", I, [P, I]), ("orcN_init_equilibrium", I, [P])]:
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self._case = to_case(hc.coarse)
        flat = []
        for lo, hi in hc.boxes:
            flat += list(lo) + list(hi)
        arr = (C.c_int * max(1, len(flat)))(*flat)
        self.h = lib.orcN_create(C.byref(self._case), self.nlev, arr)
        if not self.h:
            raise RuntimeError("orcN_create refused the level boxes")
        self.q = hc.coarse.lattice.q
        self.shapes = tuple(hc.box_case(l).shape for l in range(self.nlev))

    def level(self, lev: int):
        return self.lib.orcN_level(self.h, lev)

    def close(self):
        if self.h:
            self.lib.orcN_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_macro(self, lev, rho, ux, uy, uz=None):
        m = np.zeros((4,) + self.shapes[lev])
        m[0], m[1], m[2] = rho, ux, uy
        if uz is not None:
            m[3] = uz
        m = np.ascontiguousarray(m)
        self.lib.orc_set_macro(self.level(lev), _dp(m))

    def init_equilibrium(self):
        self.lib.orcN_init_equilibrium(self.h)

    def ib_create(self, ib):
        """The body lives on the finest level."""
        if getattr(ib, "airfoil", None) is not None:
            p = np.ascontiguousarray(np.asarray(ib.airfoil, dtype=np.float64))
            self.lib.orc_set_airfoil(_dp(p))
        self._ib = to_ib_case(ib)
        if self.lib.orc_ib_create(self.level(self.nlev - 1), C.byref(self._ib)) != 0:
            raise RuntimeError("oracle: ib_create failed")

    def step(self, n: int = 1):
        self.lib.orcN_step(self.h, int(n))

    def get_f(self, lev):
        out = np.zeros((self.q,) + self.shapes[lev])
        self.lib.orc_get_f(self.level(lev), _dp(out))
        return out

    def get_macro(self, lev):
        out = np.zeros((4,) + self.shapes[lev])
        self.lib.orc_get_macro(self.level(lev), _dp(out))
        return out

    def force_record(self):
        out = np.zeros(FORCE_REC)
        self.lib.orc_force_record(self.level(self.nlev - 1), _dp(out))
        return out

    def marker_force_sum(self):
        out = np.zeros(3)
        self.lib.orc_ib_marker_force_sum(self.level(self.nlev - 1), _dp(out))
        return out


class CpuTwoLevel(CpuHierarchy):
    """The two-level hierarchy of a ``cases.TwoLevelCase``: coarse level = the
    domain, one fine box of ratio 2."""

    class _HC:
        def __init__(self, tl):
            self.coarse, self.nlev = tl.coarse, 2
            self.boxes = ((tl.fine_lo, tl.fine_hi),)
            self._tl = tl

        def box_case(self, l):
            return self.coarse if l == 0 else self._tl.fine_box()

    def __init__(self, tl):
        self.tl = tl
        super().__init__(CpuTwoLevel._HC(tl))


def vorticity_pressure(mg, ng: int, dim: int, dx: float, dy: float, dz: float):
    """vorticityDiagnostic / visPara (Source/LBM/visPara.H:10-54) on the valid
    cells of a FillPatched macro array mg[comp, k, j, i] (comps rho, u, v, w,
    ...; ng ghost layers, none in z for 2D): (vorticity, pressure), each
    [nz, ny, nx]."""
    rho, u, v, w = mg[0], mg[1], mg[2], mg[3]
    kz = slice(ng, -ng) if dim == 3 else slice(0, 1)

    def sh(a, di=0, dj=0, dk=0):
        gz, gy, gx = a.shape
        ks = slice(ng + dk, gz - ng + dk) if dim == 3 else slice(0, 1)
        return a[ks, ng + dj:gy - ng + dj, ng + di:gx - ng + di]

    dv_dx = (sh(v, 1) - sh(v, -1)) / (2.0 * dx)
    du_dy = (sh(u, 0, 1) - sh(u, 0, -1)) / (2.0 * dy)
    if dim == 3:
        du_dz = (sh(u, 0, 0, 1) - sh(u, 0, 0, -1)) / (2.0 * dz)
        dw_dx = (sh(w, 1) - sh(w, -1)) / (2.0 * dx)
        dv_dz = (sh(v, 0, 0, 1) - sh(v, 0, 0, -1)) / (2.0 * dz)
        dw_dy = (sh(w, 0, 1) - sh(w, 0, -1)) / (2.0 * dy)
        ox, oy, oz = dw_dy - dv_dz, du_dz - dw_dx, dv_dx - du_dy
        vor = np.sqrt(ox * ox + oy * oy + oz * oz)
    else:
        vor = dv_dx - du_dy
    pres = (sh(rho) - 1.0) / 3.0
    return vor, pres


def error_est_tags(vor, threshold: float, prob_lo, prob_hi, dx, box=None, no_refine=(0.0, 0.0),
                   levelset=None):
    """ErrorEst's tagging (Source/Core/AmrCoreLBM.cpp:1073-1180 with
    vorticity_tagging and levelset_tagging, Source/Tagging.H:12-35) of
    vor[nz, ny, nx]: 0/1 tags.  levelset: None or (x0, y0, z0, R,
    n_cells_band, dx_min) of the cylinder-geometry branch, whose phi is
    LevelSetManager::build_from_cylinder (Source/LevelSet/LevelSet.cpp:36-74)."""
    nz, ny, nx = vor.shape
    k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    x = prob_lo[0] + (i + 0.5) * dx[0]
    tags = (np.abs(vor) > threshold)
    if levelset is not None:
        x0, y0, z0, R, nband, dx_min = levelset
        y = prob_lo[1] + (j + 0.5) * dx[1]
        r2 = (x - x0) * (x - x0) + (y - y0) * (y - y0)
        if nz > 1:
            z = prob_lo[2] + (k + 0.5) * dx[2]
            r2 = r2 + (z - z0) * (z - z0)
        phi = np.sqrt(r2) - R
        tags = tags | (phi < (float(int(nband)) + 0.5) * dx_min)
    if box is not None:
        y = prob_lo[1] + (j + 0.5) * dx[1]
        z = prob_lo[2] + (k + 0.5) * dx[2] if nz > 1 else np.zeros_like(x)
        inb = ((x >= box[0][0]) & (x <= box[1][0]) & (y >= box[0][1]) & (y <= box[1][1])
               & (z >= box[0][2]) & (z <= box[1][2]))
        tags = tags | inb
    if no_refine[0] > 0.0 or no_refine[1] > 0.0:
        blocked = (x <= prob_lo[0] + no_refine[0]) | (x >= prob_hi[0] - no_refine[1])
        tags = tags & ~blocked
    return tags.astype(np.uint8)
