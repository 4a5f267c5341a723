"""Level and immersed-boundary case descriptions, and the synthetic workloads.

Field names follow the reference's input keys (``amr.n_cell``,
``geometry.*``, ``amrbc.*``, ``lbmPhysicalParameters.nu``,
``lbm.prescribed_force``, ``ibm.*``; Source/Core/AmrCoreLBM.cpp:1188-1419 and
Source/IBM/MarkerIBParams.H).  Lattice units: unless a builder says otherwise
the base cell is dx = 1, so dt = dx = 1 and tau = 0.5 + 3 nu
(Source/Core/AmrCoreLBM.cpp:225-238).

The builders produce the synthetic inputs of the benchmark configurations:
no reference dataset is involved, every field is analytic or seeded.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np

from .lattice import D2Q9, D3Q19, D3Q27, Lattice

INT_DIR, FOEXTRAP, EXT_DIR, USER_1, USER_2 = 0, 2, 3, 1001, 1002


@dataclass
class LevelCase:
    lattice: Lattice
    n_cell: tuple
    prob_lo: tuple = (0.0, 0.0, 0.0)
    prob_hi: tuple | None = None
    periodic: tuple = (True, True, True)
    bc_lo: tuple = (INT_DIR, INT_DIR, INT_DIR)
    bc_hi: tuple = (INT_DIR, INT_DIR, INT_DIR)
    bc_lo_val: tuple = ((0.0,) * 4,) * 3  # per dim (rho, ux, uy, uz)
    bc_hi_val: tuple = ((0.0,) * 4,) * 3
    nu: float = 0.1
    prescribed_force: tuple | None = None
    nghost: int = 3
    name: str = "case"

    def __post_init__(self):
        n = tuple(int(x) for x in self.n_cell) + (1,) * (3 - len(self.n_cell))
        if self.lattice.dim == 2:
            n = (n[0], n[1], 1)
        self.n_cell = n
        if self.prob_hi is None:
            self.prob_hi = tuple(float(self.prob_lo[d]) + float(n[d]) for d in range(3))
        per = tuple(bool(p) for p in self.periodic) + (True,) * (3 - len(self.periodic))
        self.periodic = per

    @property
    def dim(self) -> int:
        return self.lattice.dim

    @property
    def dx(self) -> float:
        return (self.prob_hi[0] - self.prob_lo[0]) / self.n_cell[0]

    @property
    def tau(self) -> float:
        # AmrCoreLBM.cpp:225: tau_base = 3 nu / dx + 0.5
        return 3.0 * self.nu / self.dx + 0.5

    @property
    def dt(self) -> float:
        return self.dx

    @property
    def shape(self) -> tuple:
        """(nz, ny, nx) -- 2D cases have nz = 1."""
        return (self.n_cell[2], self.n_cell[1], self.n_cell[0])

    @property
    def cells(self) -> int:
        return int(np.prod(self.n_cell[: self.dim]))


@dataclass
class MarkerIB:
    """MarkerIBParams + body (ibm.x0,y0,z0,R) + force evaluation settings."""
    coupling_method: int = 1      # 0 explicit, 1 ivc (wu_shu), 2 explicit_diag
    delta_type: int = 4
    loop_ns: int = 1
    mdf_relax: float = 1.0
    explicit_diag_eps: float = 1.0e-8
    geometry_type: int = 0        # 0 cylinder/sphere, 1 box, 2 pitching NACA
    box_xlo: float = 0.0
    box_xhi: float = 0.0
    box_ylo: float = 0.0
    box_yhi: float = 0.0
    box_zlo: float = 0.0
    box_zhi: float = 0.0
    box_ds: float = 0.0
    box_lid_only: int = 0
    box_lid_ux: float = 0.0
    box_lid_uy: float = 0.0
    box_lid_uz: float = 0.0
    box_wall_tol: float = 0.0
    n_marker: int = 0
    rd: float = 0.0
    ubx: float = 0.0
    uby: float = 0.0
    ubz: float = 0.0
    omx: float = 0.0
    omy: float = 0.0
    omz: float = 0.0
    ivc_diag_reg: float = 1.3
    ivc_rebuild_matrix: int = 0
    renormalize_delta: int = 0
    x0: float = 0.0
    y0: float = 0.0
    z0: float = 0.0
    R: float = 1.0
    force_eval_method: int = 0    # 0 momentum_exchange, 1 eulerian, 2 marker
    U0: float = 0.1
    # pitching NACA (Examples/Pitching_airfoil/IBMUserDefinedGeometry.H:14-20)
    airfoil: tuple | None = None  # (chord, thickness, mean, amplitude, frequency, phase, pivot_x)
    # refinement box around the body in radii (MarkerIBParams.H:86-88; <= 0: R + padding)
    refine_upstream: float = -1.0
    refine_downstream: float = -1.0
    refine_cross: float = -1.0

    AIRFOIL_DEFAULT = (20.0, 0.12, 0.0, 0.2617993877991494, 0.0015, 0.0, 0.0)


def _bcv(rho=1.0, ux=0.0, uy=0.0, uz=0.0):
    return (float(rho), float(ux), float(uy), float(uz))


# ---------------------------------------------------------------------------
# synthetic workloads
# ---------------------------------------------------------------------------
def taylor_green(n: int = 256, U0: float = 0.01, tau: float = 0.8, lattice: Lattice = D2Q9):
    """D2Q9 Taylor-Green vortex on a periodic n x n box (lattice units)."""
    nu = (tau - 0.5) / 3.0
    case = LevelCase(lattice, (n, n, 1), periodic=(True, True, True), nu=nu, name=f"tgv{n}")

    def init():
        x = 2.0 * np.pi * (np.arange(n) + 0.5) / n
        X, Y = np.meshgrid(x, x, indexing="xy")  # [j, i]
        u = U0 * np.sin(X) * np.cos(Y)
        v = -U0 * np.cos(X) * np.sin(Y)
        p = -(U0 ** 2 / 4.0) * (np.cos(2 * X) + np.cos(2 * Y))
        rho = 1.0 + 3.0 * p
        sh = (1, n, n)
        return rho.reshape(sh), u.reshape(sh), v.reshape(sh), np.zeros(sh)

    return case, init


def uniform_init(case: LevelCase, rho=1.0, u=(0.0, 0.0, 0.0)):
    def init():
        sh = case.shape
        return (np.full(sh, rho), np.full(sh, u[0]), np.full(sh, u[1]), np.full(sh, u[2]))
    return init


def cylinder(nx=1024, ny=512, D=40.0, center=(256.0, 256.0), U=0.05, Re=100.0, dx=1.0,
             coupling=1, n_marker=0, inflow_uy=0.0):
    """2D flow past a cylinder: ext_dir inflow (rho=1, u=U) at x-lo,
    foextrap outflow at x-hi, periodic in y, marker IBM with IVC coupling.
    `inflow_uy` is the inflow's transverse velocity (the deck's
    amrbc.bc_lo_0_uy_val, 1e-4 in Examples/Cylinder_flow/inputs), which breaks
    the symmetry so that the wake starts shedding within the run."""
    nu = U * D / Re
    case = LevelCase(D2Q9, (nx, ny, 1), prob_hi=(nx * dx, ny * dx, 1.0),
                     periodic=(False, True, True), bc_lo=(EXT_DIR, INT_DIR, INT_DIR),
                     bc_hi=(FOEXTRAP, INT_DIR, INT_DIR),
                     bc_lo_val=(_bcv(1.0, U, inflow_uy), _bcv(0.0), _bcv(0.0)), nu=nu,
                     name=f"cylinder{nx}x{ny}")
    ib = MarkerIB(coupling_method=coupling, delta_type=4, loop_ns=1, ivc_diag_reg=1.3,
                  x0=center[0], y0=center[1], R=D / 2.0, U0=U, n_marker=n_marker)
    return case, ib, uniform_init(case, 1.0, (U, 0.0, 0.0))


def sphere(nx=256, ny=128, nz=128, D=32.0, center=(64.0, 64.0, 64.0), U=0.04, Re=100.0,
           lattice: Lattice = D3Q19, coupling=1, n_marker=0):
    """3D flow past a sphere: ext_dir inflow at x-lo, foextrap at x-hi,
    periodic in y and z, golden-spiral markers (IBMarkerDF.cpp:385-421)."""
    nu = U * D / Re
    case = LevelCase(lattice, (nx, ny, nz), periodic=(False, True, True),
                     bc_lo=(EXT_DIR, INT_DIR, INT_DIR), bc_hi=(FOEXTRAP, INT_DIR, INT_DIR),
                     bc_lo_val=(_bcv(1.0, U), _bcv(0.0), _bcv(0.0)), nu=nu,
                     name=f"sphere{nx}x{ny}x{nz}")
    ib = MarkerIB(coupling_method=coupling, delta_type=4, loop_ns=1, ivc_diag_reg=1.3,
                  x0=center[0], y0=center[1], z0=center[2], R=D / 2.0, U0=U, n_marker=n_marker)
    return case, ib, uniform_init(case, 1.0, (U, 0.0, 0.0))


def square_duct(N=32, L=8, force=1.0e-5, nu=0.06, lattice: Lattice = D3Q19):
    """Body-force driven laminar square duct (Examples/SquareDuct_flow/inputs):
    x periodic (length L), face-mirrored user_2 walls on y and z."""
    case = LevelCase(lattice, (L, N, N), prob_lo=(0.0, -N / 2.0, -N / 2.0),
                     prob_hi=(float(L), N / 2.0, N / 2.0), periodic=(True, False, False),
                     bc_lo=(INT_DIR, USER_2, USER_2), bc_hi=(INT_DIR, USER_2, USER_2),
                     bc_lo_val=(_bcv(0.0), _bcv(1.0), _bcv(1.0)),
                     bc_hi_val=(_bcv(0.0), _bcv(1.0), _bcv(1.0)), nu=nu,
                     prescribed_force=(force, 0.0, 0.0), name=f"duct{N}")
    return case, uniform_init(case)


def couette(n=64, U=0.1, nu=0.064):
    """Couette flow (Examples/Couette_flow/inputs): foextrap in x, ext_dir
    walls in y (lid velocity U at y-hi)."""
    case = LevelCase(D2Q9, (n, n, 1), periodic=(False, False, True),
                     bc_lo=(FOEXTRAP, EXT_DIR, INT_DIR), bc_hi=(FOEXTRAP, EXT_DIR, INT_DIR),
                     bc_lo_val=(_bcv(0.0), _bcv(1.0, 0.0), _bcv(0.0)),
                     bc_hi_val=(_bcv(0.0), _bcv(1.0, U), _bcv(0.0)), nu=nu, name=f"couette{n}")
    return case, uniform_init(case)


def channel_bounce_back(nx=32, ny=24, force=1.0e-5, nu=0.1):
    """Force-driven channel: x periodic, halfway bounce-back (user_1) walls in y."""
    case = LevelCase(D2Q9, (nx, ny, 1), periodic=(True, False, True),
                     bc_lo=(INT_DIR, USER_1, INT_DIR), bc_hi=(INT_DIR, USER_1, INT_DIR),
                     bc_lo_val=(_bcv(0.0), _bcv(1.0), _bcv(0.0)),
                     bc_hi_val=(_bcv(0.0), _bcv(1.0), _bcv(0.0)), nu=nu,
                     prescribed_force=(force, 0.0, 0.0), name=f"channel{nx}x{ny}")
    return case, uniform_init(case)


def cavity_lid(n=64, U=0.1, nu=0.064):
    """Lid-driven cavity with a marker box lid (Examples/Cavity_flow/inputs_ibm_box style)."""
    case = LevelCase(D2Q9, (n, n, 1), periodic=(False, False, True),
                     bc_lo=(USER_1, USER_1, INT_DIR), bc_hi=(USER_1, USER_1, INT_DIR),
                     bc_lo_val=(_bcv(1.0), _bcv(1.0), _bcv(0.0)),
                     bc_hi_val=(_bcv(1.0), _bcv(1.0), _bcv(0.0)), nu=nu, name=f"cavity{n}")
    ib = MarkerIB(coupling_method=0, delta_type=4, loop_ns=2, geometry_type=1, box_lid_only=1,
                  box_lid_ux=U, box_xlo=0.0, box_xhi=float(n), box_ylo=0.0, box_yhi=float(n) - 2.0,
                  U0=U)
    return case, ib, uniform_init(case)


def pitching_airfoil(nx=512, ny=256, chord=64.0, pivot=(128.0, 128.0), U=0.05, Re=100.0,
                     amplitude_deg=10.0, reduced_frequency=0.1, quarter_chord=True,
                     thickness=0.12):
    """2D NACA 00xx pitching about its quarter chord (user-defined marker
    geometry, Examples/Pitching_airfoil/IBMUserDefinedGeometry.H; the pivot is
    moved from the leading edge to c/4).  k = omega c / (2 U)."""
    nu = U * chord / Re
    omega = 2.0 * U * reduced_frequency / chord
    freq = omega / (2.0 * math.pi)
    case = LevelCase(D2Q9, (nx, ny, 1), periodic=(False, True, True),
                     bc_lo=(EXT_DIR, INT_DIR, INT_DIR), bc_hi=(FOEXTRAP, INT_DIR, INT_DIR),
                     bc_lo_val=(_bcv(1.0, U), _bcv(0.0), _bcv(0.0)), nu=nu,
                     name=f"airfoil{nx}x{ny}")
    ib = MarkerIB(coupling_method=1, delta_type=4, loop_ns=1, geometry_type=2,
                  ivc_diag_reg=1.3, x0=pivot[0], y0=pivot[1], R=chord / 2.0, U0=U,
                  airfoil=(chord, thickness, 0.0, math.radians(amplitude_deg), freq, 0.0,
                           0.25 * chord if quarter_chord else 0.0))
    return case, ib, uniform_init(case, 1.0, (U, 0.0, 0.0))


def batch_mix(n_cases: int = 64, seed: int = 20261203, U: float = 0.05):
    """The batched D2Q9 workload: n_cases independent single-level cases with
    seeded grid sizes from 256 x 128 to 1024 x 512 (multiples of 8), each a
    cylinder (D uniform in [16, 48] cells, Re uniform in [20, 200]) or a NACA
    0012 pitching about its quarter chord (chord uniform in [64, 128] cells,
    amplitude uniform in [2, 15] degrees, reduced frequency uniform in
    [0.05, 0.3], Re 100), inflow U.  Returns (case, ib, init) triples."""
    rng = np.random.default_rng(seed)
    out = []
    for c in range(n_cases):
        nx = int(rng.integers(256 // 8, 1024 // 8 + 1)) * 8
        ny = int(rng.integers(128 // 8, 512 // 8 + 1)) * 8
        if rng.random() < 0.5:
            D = float(rng.uniform(16.0, 48.0))
            D = min(D, 0.3 * ny)
            Re = float(rng.uniform(20.0, 200.0))
            cx, cy = 0.25 * nx + 0.37, 0.5 * ny - 0.21
            case, ib, init = cylinder(nx=nx, ny=ny, D=D, center=(cx, cy), U=U, Re=Re)
        else:
            chord = float(rng.uniform(64.0, 128.0))
            chord = min(chord, 0.45 * nx, 0.9 * ny)
            amp = float(rng.uniform(2.0, 15.0))
            k = float(rng.uniform(0.05, 0.3))
            px, py = 0.25 * nx + 0.37, 0.5 * ny - 0.21
            case, ib, init = pitching_airfoil(nx=nx, ny=ny, chord=chord, pivot=(px, py), U=U,
                                              Re=100.0, amplitude_deg=amp, reduced_frequency=k)
        case.name = f"{case.name}#{c}"
        out.append((case, ib, init))
    return out


# ---------------------------------------------------------------------------
# static two-level hierarchies (amr.max_level = 1, amr.ref_ratio = 2)
# ---------------------------------------------------------------------------
@dataclass
class TwoLevelCase:
    """A coarse level equal to the domain and one fixed fine box of
    refinement ratio 2 (fine-domain cell indices, lo even, hi odd, at least
    two coarse cells inside every face of the domain).  The fine level is
    stepped twice per coarse step (timeStepWithSubcycling,
    Source/Core/AmrCoreLBM.cpp:1690-1755); a body lives on it (the finest
    level, AdvanceLBMAtLevel.cpp:30, 73-93)."""
    coarse: LevelCase
    fine_lo: tuple
    fine_hi: tuple
    name: str = "two_level"

    def __post_init__(self):
        d = self.coarse.dim
        lo = tuple(int(v) for v in self.fine_lo) + (0,) * (3 - len(self.fine_lo))
        hi = tuple(int(v) for v in self.fine_hi) + (0,) * (3 - len(self.fine_hi))
        self.fine_lo, self.fine_hi = lo[:3], hi[:3]
        for a in range(d):
            if self.fine_lo[a] % 2 or self.fine_hi[a] % 2 == 0 or self.fine_hi[a] < self.fine_lo[a]:
                raise ValueError("fine box must cover whole coarse cells (lo even, hi odd)")
            if self.fine_lo[a] // 2 < 2 or self.fine_hi[a] // 2 > self.coarse.n_cell[a] - 3:
                raise ValueError("fine box must lie two coarse cells inside the domain")

    @property
    def dim(self) -> int:
        return self.coarse.dim

    @property
    def fine_n_cell(self) -> tuple:
        return tuple((self.fine_hi[a] - self.fine_lo[a] + 1) if a < self.dim else 1 for a in range(3))

    def fine_level(self) -> LevelCase:
        """The fine level's domain (twice the coarse cells, same geometry)."""
        c = self.coarse
        n = tuple(2 * c.n_cell[a] if a < c.dim else 1 for a in range(3))
        return replace(c, n_cell=n, name=c.name + "_fine")

    def fine_box(self) -> LevelCase:
        """The fine box as a level of its own (its cells and physical extent),
        for initial fields evaluated at its cell centres."""
        c = self.coarse
        dxf = c.dx / 2.0
        lo = tuple(c.prob_lo[a] + dxf * self.fine_lo[a] if a < c.dim else c.prob_lo[a] for a in range(3))
        hi = tuple(c.prob_lo[a] + dxf * (self.fine_hi[a] + 1) if a < c.dim else c.prob_hi[a]
                   for a in range(3))
        return replace(c, n_cell=self.fine_n_cell, prob_lo=lo, prob_hi=hi, periodic=(False,) * 3,
                       name=c.name + "_finebox")


def field_init(case: LevelCase, fn):
    """Initial (rho, u, v, w) of fn(x, y, z) at the cell centres of a level."""
    def init():
        nz, ny, nx = case.shape
        dx = case.dx
        x = case.prob_lo[0] + (np.arange(nx) + 0.5) * dx
        y = case.prob_lo[1] + (np.arange(ny) + 0.5) * dx
        z = case.prob_lo[2] + (np.arange(nz) + 0.5) * dx if case.dim == 3 else np.zeros(1)
        Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
        return tuple(np.asarray(v, dtype=np.float64) * np.ones(case.shape) for v in fn(X, Y, Z))
    return init


def shear_layer_two_level(n=64, U0=0.02, nu=0.01, fine=(24, 48), lattice: Lattice = D2Q9):
    """Periodic box with a perturbed double shear layer and a centred fine
    patch covering fine cells [fine[0], fine[1]) in every direction (no body):
    velocity gradients cross the coarse-fine boundary."""
    periodic = (True, True, True)
    dims = (n, n, n if lattice.dim == 3 else 1)
    coarse = LevelCase(lattice, dims, periodic=periodic, nu=nu, name=f"shear{n}")
    lo = (fine[0],) * lattice.dim
    hi = (fine[1] - 1,) * lattice.dim
    tl = TwoLevelCase(coarse, lo, hi, name=f"shear{n}_2lev")
    L = float(n)

    def fn(X, Y, Z):
        u = U0 * np.tanh(30.0 * (np.abs(Y / L - 0.5) - 0.25))
        v = 0.05 * U0 * np.sin(2.0 * np.pi * X / L)
        w = 0.02 * U0 * np.sin(2.0 * np.pi * Z / L) if lattice.dim == 3 else 0.0 * X
        return 1.0 + 0.0 * X, u, v, w

    return tl, field_init(coarse, fn), field_init(tl.fine_box(), fn)


def cylinder_two_level(nx=256, ny=128, D=24.0, center=(64.3, 63.7), U=0.05, Re=100.0,
                       upstream=1.0, downstream=4.0, cross=1.5):
    """The reference's 2D cylinder deck on two levels (Examples/Cylinder_flow/
    inputs: max_level 1, ref_ratio 2): coarse level as ``cylinder``, a fine box
    around the body and its near wake (upstream / downstream / cross extents
    in diameters from the centre) on which the marker IBM runs, with the
    body's cells at twice the resolution."""
    case, ib, init_c = cylinder(nx=nx, ny=ny, D=D, center=center, U=U, Re=Re)
    lo = [int(math.floor((center[0] - upstream * D))) * 2, int(math.floor((center[1] - cross * D))) * 2]
    hi = [int(math.ceil((center[0] + downstream * D))) * 2 - 1,
          int(math.ceil((center[1] + cross * D))) * 2 - 1]
    lo = [max(lo[a], 4) for a in range(2)]
    hi = [min(hi[a], 2 * (case.n_cell[a] - 2) - 1) for a in range(2)]
    tl = TwoLevelCase(case, tuple(lo), tuple(hi), name=f"cylinder{nx}x{ny}_2lev")
    init_f = uniform_init(tl.fine_box(), 1.0, (U, 0.0, 0.0))
    return tl, ib, init_c, init_f


def sphere_two_level(nx=256, ny=128, nz=128, D=32.0, center=(64.0, 64.0, 64.0), U=0.04, Re=100.0,
                     box_lo=(32, 32, 32), box_hi=(128, 96, 96), lattice: Lattice = D3Q19):
    """The D3Q19 sphere on two levels: base grid as ``sphere`` plus one
    refined level (ratio 2) over the base-cell box [box_lo, box_hi) around
    the sphere, on which the marker IBM runs with markers about one fine cell
    apart (golden-spiral lattice, IBMarkerDF.cpp:385-421: ~4 pi R^2 / dx_f^2
    points, 12.9k for D = 32 base cells)."""
    case, ib, init_c = sphere(nx, ny, nz, D=D, center=center, U=U, Re=Re, lattice=lattice)
    lo = tuple(2 * int(v) for v in box_lo)
    hi = tuple(2 * int(v) - 1 for v in box_hi)
    tl = TwoLevelCase(case, lo, hi, name=f"sphere{nx}x{ny}x{nz}_2lev")
    init_f = uniform_init(tl.fine_box(), 1.0, (U, 0.0, 0.0))
    return tl, ib, init_c, init_f


@dataclass
class HierarchyCase:
    """A coarse level equal to the domain and one fixed box on each finer
    level (refinement ratio 2 between levels): ``boxes[l - 1]`` = (lo, hi) of
    level l in that level's own cell indices (lo even, hi odd; coarsened, at
    least two cells inside the box of level l - 1, or inside the domain for
    level 1).  Each level steps twice per step of the level above
    (timeStepWithSubcycling, Source/Core/AmrCoreLBM.cpp:1690-1755); a body
    lives on the finest level."""
    coarse: LevelCase
    boxes: tuple
    name: str = "hierarchy"

    def __post_init__(self):
        d = self.coarse.dim
        norm = []
        for lo, hi in self.boxes:
            lo = tuple(int(v) for v in lo) + (0,) * (3 - len(lo))
            hi = tuple(int(v) for v in hi) + (0,) * (3 - len(hi))
            norm.append((lo[:3], hi[:3]))
        self.boxes = tuple(norm)
        for l in range(1, self.nlev):
            lo, hi = self.boxes[l - 1]
            plo, phi = self.box_lohi(l - 1)
            for a in range(d):
                if lo[a] % 2 or hi[a] % 2 == 0 or hi[a] < lo[a]:
                    raise ValueError(f"level {l}: the box must cover whole cells of level {l - 1}")
                if lo[a] // 2 < plo[a] + 2 or hi[a] // 2 > phi[a] - 2:
                    raise ValueError(f"level {l}: the box must lie two cells inside level {l - 1}'s box")

    @property
    def nlev(self) -> int:
        return 1 + len(self.boxes)

    @property
    def dim(self) -> int:
        return self.coarse.dim

    def box_lohi(self, l: int):
        if l == 0:
            c = self.coarse
            return (0, 0, 0), tuple(c.n_cell[a] - 1 if a < c.dim else 0 for a in range(3))
        return self.boxes[l - 1]

    def n_cell_of(self, l: int) -> tuple:
        lo, hi = self.box_lohi(l)
        return tuple((hi[a] - lo[a] + 1) if a < self.dim else 1 for a in range(3))

    def level_case(self, l: int) -> LevelCase:
        """Level l's whole domain (2^l times the coarse cells, same geometry)."""
        c = self.coarse
        n = tuple((2 ** l) * c.n_cell[a] if a < c.dim else 1 for a in range(3))
        return replace(c, n_cell=n, name=f"{c.name}_lev{l}")

    def box_case(self, l: int) -> LevelCase:
        """Level l's box as a level of its own (its cells and physical extent),
        for initial fields evaluated at its cell centres."""
        c = self.coarse
        if l == 0:
            return c
        lo, hi = self.boxes[l - 1]
        dx = c.dx / (2 ** l)
        plo = tuple(c.prob_lo[a] + dx * lo[a] if a < c.dim else c.prob_lo[a] for a in range(3))
        phi = tuple(c.prob_lo[a] + dx * (hi[a] + 1) if a < c.dim else c.prob_hi[a] for a in range(3))
        return replace(c, n_cell=self.n_cell_of(l), prob_lo=plo, prob_hi=phi, periodic=(False,) * 3,
                       name=f"{c.name}_box{l}")

    def cells(self, l: int) -> int:
        return int(np.prod(self.n_cell_of(l)[: self.dim]))

    def updates_per_coarse_step(self) -> int:
        """Cell updates of one coarse step: level l steps 2^l times."""
        return sum((2 ** l) * self.cells(l) for l in range(self.nlev))


def nested_boxes(finest_lo, finest_hi, nlev: int, n_cell, dim: int, grow: int = 8):
    """Boxes of levels 1 .. nlev - 1 around a finest-level box (given in the
    finest level's indices): each coarser box is the finer one coarsened and
    grown by `grow` cells, aligned to whole cells of the level above."""
    L = nlev - 1
    boxes = [None] * L
    lo = [int(v) for v in finest_lo[:dim]]
    hi = [int(v) for v in finest_hi[:dim]]
    lo = [v - (v % 2) for v in lo]
    hi = [v + (1 - v % 2) for v in hi]
    boxes[L - 1] = (tuple(lo), tuple(hi))
    for l in range(L - 1, 0, -1):
        lo = [v // 2 - grow for v in lo]
        hi = [v // 2 + grow for v in hi]
        lo = [v - (v % 2) for v in lo]
        hi = [v + (1 - v % 2) for v in hi]
        boxes[l - 1] = (tuple(lo), tuple(hi))
    # keep level 1 two coarse cells inside the domain
    lo1, hi1 = boxes[0]
    for a in range(dim):
        if lo1[a] // 2 < 2 or hi1[a] // 2 > n_cell[a] - 3:
            raise ValueError("the refined boxes reach the domain boundary; use a larger domain")
    return tuple(boxes)


def cylinder_hierarchy(nx=1024, ny=512, D=40.0, center=(256.0, 256.0), U=0.05, Re=100.0, nlev=3,
                       upstream=1.0, downstream=4.0, cross=1.5, grow=8, inflow_uy=0.0):
    """The reference's 2D cylinder deck on nlev levels (Examples/Cylinder_flow/
    inputs, ref_ratio 2): coarse level as ``cylinder``; the finest box around
    the body and its near wake (upstream / downstream / cross extents in
    diameters from the centre), every level in between the finer box
    coarsened and grown by `grow` of its cells.  The marker IBM runs on the
    finest level with markers about one finest cell apart."""
    case, ib, init_c = cylinder(nx=nx, ny=ny, D=D, center=center, U=U, Re=Re, inflow_uy=inflow_uy)
    r = 2 ** (nlev - 1)
    dx = case.dx
    flo = [int(math.floor((center[0] - upstream * D) / dx * r)), int(math.floor((center[1] - cross * D) / dx * r))]
    fhi = [int(math.ceil((center[0] + downstream * D) / dx * r)) - 1,
           int(math.ceil((center[1] + cross * D) / dx * r)) - 1]
    boxes = nested_boxes(flo, fhi, nlev, case.n_cell, 2, grow)
    hc = HierarchyCase(case, boxes, name=f"cylinder{nx}x{ny}_{nlev}lev")
    inits = [init_c] + [uniform_init(hc.box_case(l), 1.0, (U, 0.0, 0.0)) for l in range(1, nlev)]
    return hc, ib, inits


def shear_layer_hierarchy(n=64, U0=0.02, nu=0.01, nlev=3, lattice: Lattice = D2Q9):
    """Periodic box with a perturbed double shear layer and nested boxes
    around its centre on every finer level (no body): velocity gradients
    cross every coarse-fine boundary."""
    dims = (n, n, n if lattice.dim == 3 else 1)
    coarse = LevelCase(lattice, dims, periodic=(True, True, True), nu=nu, name=f"shear{n}")
    L = nlev - 1
    r = 2 ** L
    c = n * r // 2
    half = n * r // 8
    boxes = nested_boxes([c - half] * lattice.dim, [c + half - 1] * lattice.dim, nlev, dims,
                         lattice.dim, grow=4)
    hc = HierarchyCase(coarse, boxes, name=f"shear{n}_{nlev}lev")
    Lx = float(n)

    def fn(X, Y, Z):
        u = U0 * np.tanh(30.0 * (np.abs(Y / Lx - 0.5) - 0.25))
        v = 0.05 * U0 * np.sin(2.0 * np.pi * X / Lx)
        w = 0.02 * U0 * np.sin(2.0 * np.pi * Z / Lx) if lattice.dim == 3 else 0.0 * X
        return 1.0 + 0.0 * X, u, v, w

    return hc, [field_init(hc.box_case(l), fn) for l in range(nlev)]
