"""Parity of the sm_100a library (through the C ABI) with the CPU oracle.

Tolerances:
* FP64 storage, no immersed boundary: bit-exact (the kernels keep the
  reference's operation order with separately rounded products and sums);
* FP64 with the marker IB: relative L2 <= 1e-12 in populations and macro
  fields (the IVC system is solved by CG to 1e-14 instead of a dense LU, and
  spreading sums in atomic order);
* FP32 shifted / FP16 scaled storage: stated per test against the FP64 oracle.
"""
import ctypes as C

import numpy as np
import pytest

from ilbmrex_b200 import capi, cases
from oracle.checker import CpuLevel
from tests.golden.golden_cases import GOLDEN_CASES

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.level import LevelSolver  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def _pair(name, storage="f64", steps=None):
    builder, nsteps = GOLDEN_CASES[name]
    steps = steps or nsteps
    case, init, ib = builder()
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    if ib is not None:
        cpu.ib_create(ib)
    cpu.step(steps)
    gpu = LevelSolver(case, storage, ib=ib)
    gpu.set_macro(*init())
    gpu.step(steps, record_force=ib is not None)
    return cpu, gpu, ib


NO_IB = [n for n in sorted(GOLDEN_CASES) if GOLDEN_CASES[n][0]()[2] is None]
WITH_IB = [n for n in sorted(GOLDEN_CASES) if GOLDEN_CASES[n][0]()[2] is not None]


@pytest.mark.parametrize("name", NO_IB)
def test_fp64_bit_exact(name):
    cpu, gpu, _ = _pair(name)
    np.testing.assert_array_equal(gpu.get_f(), cpu.get_f())
    np.testing.assert_array_equal(gpu.get_macro(), cpu.get_macro())
    assert gpu.ctx.launches() > 0
    gpu.close()


def _order_sensitivity(name):
    """How far the oracle's own result moves when only the marker order of
    its force spreading is reversed: relative L2 of f, rho, u and the force
    field, and the largest relative change of Cd / Cl."""
    from oracle import checker
    builder, steps = GOLDEN_CASES[name]
    out = []
    for rev in (False, True):
        checker.set_spread_order(rev)
        try:
            case, init, ib = builder()
            c = CpuLevel(case, "oracle")
            c.set_macro(*init())
            c.init_equilibrium()
            c.ib_create(ib)
            c.step(steps)
            out.append((c.get_f(), c.get_macro(), c.get_force(), c.force_record()))
        finally:
            checker.set_spread_order(False)
    (fa, ma, Fa, ra), (fb, mb, Fb, rb) = out
    return {"f": rel_l2(fb, fa), "rho": rel_l2(mb[0], ma[0]), "u": rel_l2(mb[1:3], ma[1:3]),
            "force": rel_l2(Fb, Fa), "cdcl": float(np.max(np.abs(rb[3:5] - ra[3:5]) / np.abs(ra[3])))}


EXPLICIT = [n for n in WITH_IB if GOLDEN_CASES[n][0]()[2].coupling_method in (0, 2)]


@pytest.mark.parametrize("name", EXPLICIT)
def test_fp64_explicit_coupling_bit_exact(name):
    """Explicit and explicit_diag coupling of a body whose markers do not move:
    interpolation sums each stencil in the reference's order and spreading
    adds the markers to each cell in marker order, so the FP64 populations,
    macro fields and forces equal the reference build's bit for bit."""
    cpu, gpu, ib = _pair(name)
    np.testing.assert_array_equal(gpu.get_f(), cpu.get_f())
    np.testing.assert_array_equal(gpu.get_macro(), cpu.get_macro())
    np.testing.assert_array_equal(gpu.get_force(), cpu.get_force())
    gpu.close()


@pytest.mark.parametrize("name", WITH_IB)
def test_fp64_ib_parity(name):
    """relative L2 <= 1e-12 (force field 1e-11, Cd / Cl 1e-9), or four times
    the change the oracle itself shows when only its spreading order is
    reversed, where that is larger: the explicit_diag coupling divides the
    velocity defect by the small diagonal of the interpolation-spreading
    operator, which amplifies summation-order rounding (1e-10 relative for
    the reference's own cylinder case), and the device spreads with FP64
    atomics in an unspecified order."""
    cpu, gpu, ib = _pair(name)
    sens = _order_sensitivity(name)
    tol = lambda base, key: max(base, 4.0 * sens[key])
    assert gpu.num_markers() == cpu.num_markers()
    assert rel_l2(gpu.get_f(), cpu.get_f()) <= tol(1e-12, "f")
    mg, mc = gpu.get_macro(), cpu.get_macro()
    assert rel_l2(mg[0], mc[0]) <= tol(1e-12, "rho")
    assert rel_l2(mg[1:3], mc[1:3]) <= tol(1e-12, "u")
    assert rel_l2(gpu.get_force(), cpu.get_force()) <= tol(1e-11, "force")
    rg, rc = gpu.rec, cpu.force_record()
    np.testing.assert_allclose(rg[3:5], rc[3:5], rtol=tol(1e-9, "cdcl"), atol=1e-12)
    np.testing.assert_allclose(gpu.marker_force_sum(), cpu.marker_force_sum(), rtol=tol(1e-9, "cdcl"),
                               atol=1e-14)
    gpu.close()



def test_fp64_against_golden_fixture():
    """the committed fixtures hold the reference build's own outputs"""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / "tgv32_d2q9.npz")
    cpu, gpu, _ = _pair("tgv32_d2q9")
    np.testing.assert_array_equal(gpu.get_f(), g["f"])
    np.testing.assert_array_equal(gpu.get_macro(), g["macro"])
    gpu.close()


@pytest.mark.parametrize("storage,tol", [("f32", 2e-5), ("f16", 5e-3)])
def test_reduced_precision_taylor_green(storage, tol):
    """Velocity error against the FP64 oracle after 200 steps of TGV 64^2."""
    case, init = cases.taylor_green(64, U0=0.01, tau=0.8)
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.step(200)
    gpu = LevelSolver(case, storage)
    gpu.set_macro(*init())
    gpu.step(200)
    mg, mc = gpu.get_macro(), cpu.get_macro()
    err = rel_l2(mg[1:3], mc[1:3])
    assert err <= tol, err
    assert rel_l2(mg[0], mc[0]) <= tol
    gpu.close()


@pytest.mark.parametrize("storage,tol", [("f32", 1e-4), ("f16", 2e-2)])
def test_reduced_precision_cylinder_drag(storage, tol):
    """Cd of the FP32 / FP16 storage forms against the FP64 oracle."""
    case, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.ib_create(ib)
    cpu.step(40)
    gpu = LevelSolver(case, storage, ib=ib)
    gpu.set_macro(*init())
    gpu.step(40, record_force=True)
    rc, rg = cpu.force_record(), gpu.rec
    assert abs(rg[3] - rc[3]) <= tol * abs(rc[3]), (rg[3], rc[3])
    gpu.close()


@pytest.mark.parametrize("storage,tol", [("f32", 1e-4), ("f16", 2e-2)])
def test_reduced_precision_pitching_airfoil(storage, tol):
    """A moving body in the 4- and 2-byte forms against the FP64 oracle: its
    IVC operator is rebuilt and spread every step from the weight table the
    warp-parallel interpolation stores (the FP64 form evaluates the kernel
    in the reference's order instead).  Cd and the velocity field."""
    case, init, ib = GOLDEN_CASES["airfoil96x64_pitching_ivc"][0]()
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.ib_create(ib)
    cpu.step(20)
    gpu = LevelSolver(case, storage, ib=ib)
    gpu.set_macro(*init())
    gpu.step(20, record_force=True)
    rc, rg = cpu.force_record(), gpu.rec
    assert abs(rg[3] - rc[3]) <= tol * abs(rc[3]), (rg[3], rc[3])
    mg, mc = gpu.get_macro(), cpu.get_macro()
    scale = np.abs(mc[1:3]).max()
    assert np.abs(mg[1:3] - mc[1:3]).max() <= tol * scale
    gpu.close()


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_d3q27_duct(storage):
    """D3Q27 (the reference's sphere deck lattice) through the same kernels."""
    case, init = cases.square_duct(N=10, L=3, force=1e-5, nu=0.06, lattice=cases.D3Q27)
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.step(12)
    gpu = LevelSolver(case, storage)
    gpu.set_macro(*init())
    gpu.step(12)
    if storage == "f64":
        np.testing.assert_array_equal(gpu.get_f(), cpu.get_f())
    else:
        assert rel_l2(gpu.get_f(), cpu.get_f()) < 1e-6
    gpu.close()


@pytest.mark.parametrize("solver", [capi.IVC_CG, capi.IVC_DENSE])
def test_ivc_solvers_sphere_3d(solver):
    """3D sphere with more than 1024 markers: the grid-wide CG and the stored
    inverse both against the oracle's dense LU (relative L2 <= 1e-12)."""
    case, ib, init = cases.sphere(48, 40, 40, D=20.0, center=(16.3, 19.8, 20.1), U=0.04, Re=40.0)
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.ib_create(ib)
    cpu.step(4)
    gpu = LevelSolver(case, "f64", ib=ib)
    gpu.set_ivc_solver(solver)
    gpu.set_macro(*init())
    gpu.step(4, record_force=True)
    assert gpu.num_markers() == cpu.num_markers() > 1024
    assert rel_l2(gpu.get_f(), cpu.get_f()) <= 1e-12
    assert rel_l2(gpu.get_force(), cpu.get_force()) <= 1e-11
    np.testing.assert_allclose(gpu.marker_force_sum(), cpu.marker_force_sum(), rtol=1e-9, atol=1e-14)
    it = gpu.cg_iterations()
    assert (it > 0) if solver == capi.IVC_CG else (it == 0)
    gpu.close()


def test_ivc_dense_refused_for_moving_markers():
    from tests.golden.golden_cases import GOLDEN_CASES as G
    case, init, ib = G["airfoil96x64_pitching_ivc"][0]()
    gpu = LevelSolver(case, "f64", ib=ib)
    with pytest.raises(capi.IlbmError):
        gpu.set_ivc_solver(capi.IVC_DENSE)
    gpu.set_ivc_solver(capi.IVC_CG)
    gpu.close()


def test_momentum_exchange_matches_oracle():
    case, init = cases.taylor_green(48, U0=0.02, tau=0.7)
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.step(5)
    gpu = LevelSolver(case, "f64")
    gpu.set_macro(*init())
    gpu.step(5)
    for one_sided in (False, True):
        a = gpu.momentum_exchange(20.3, 24.1, 0.0, 7.5, one_sided)
        b = cpu.momentum_exchange(20.3, 24.1, 0.0, 7.5, one_sided)
        np.testing.assert_allclose(a, b, rtol=1e-12, atol=1e-15)
    gpu.close()


def test_caller_filled_ghosts_two_boxes():
    """AMReX drop-in mode: the level is split into two boxes whose ghost cells
    are filled by the caller (here: the oracle's FillPatch of f and macro);
    the result must equal the single-box self-fill step bit for bit."""
    case, ib, init = cases.cylinder(nx=40, ny=24, D=8, center=(12.2, 11.7), U=0.05, Re=20)
    ib = None
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.step(3)
    ng = case.nghost
    nx, ny = case.n_cell[0], case.n_cell[1]
    gx, gy = nx + 2 * ng, ny + 2 * ng
    fg = cpu.fill_patch_f().reshape(case.lattice.q, gy, gx)
    mg = cpu.fill_patch_macro().reshape(6, gy, gx)
    cpu.step(1)
    ref_f = cpu.get_f()
    from ilbmrex_b200.level import Context, level_params
    ctx = Context(case.lattice, "f64")
    L = ctx.L
    p = level_params(case, uniform_force=True)
    p.ghost_mode = capi.GHOST_CALLER
    cut = nx // 2
    boxes_lohi = [(0, cut - 1), (cut, nx - 1)]
    lb = (C.c_int * 12)(0, 0, 0, cut - 1, ny - 1, 0, cut, 0, 0, nx - 1, ny - 1, 0)
    p.level_boxes = C.cast(lb, C.POINTER(C.c_int))
    p.nlevel_boxes = 2
    dev = torch.device("cuda", 0)
    keep = []
    bx = (capi.Box_t * 2)()
    for n, (a, b) in enumerate(boxes_lohi):
        w = b - a + 1
        fin = torch.tensor(fg[:, :, a - 1 + ng:b + 2 + ng][:, ng - 1:ng + ny + 1, :], dtype=torch.float64, device=dev).contiguous()
        fout = torch.zeros_like(fin)
        mac = torch.tensor(mg[:4, :, a - 1 + ng:b + 2 + ng][:, ng - 1:ng + ny + 1, :], dtype=torch.float64, device=dev).contiguous()
        keep += [fin, fout, mac]
        B = bx[n]
        B.lo[0], B.lo[1], B.lo[2] = a, 0, 0
        B.hi[0], B.hi[1], B.hi[2] = b, ny - 1, 0
        B.ngrow_f = B.ngrow_m = 1
        B.fstride[0], B.fstride[1], B.fstride[2] = w + 2, (w + 2) * (ny + 2), (w + 2) * (ny + 2)
        B.mstride[0], B.mstride[1], B.mstride[2] = w + 2, (w + 2) * (ny + 2), (w + 2) * (ny + 2)
        B.f_in, B.f_out, B.macro_in = fin.data_ptr(), fout.data_ptr(), mac.data_ptr()
    torch.cuda.synchronize()
    capi.check(L.ilbm_level_step(ctx.h, bx, 2, C.byref(p)), "level_step caller mode")
    ctx.sync()
    got = np.zeros_like(ref_f)
    for n, (a, b) in enumerate(boxes_lohi):
        fo = keep[3 * n + 1].cpu().numpy()
        got[:, 0, :, a:b + 1] = fo[:, 1:1 + ny, 1:1 + (b - a + 1)]
    np.testing.assert_array_equal(got, ref_f)
    ctx.close()


def test_force_integral_is_deterministic():
    case, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    gpu = LevelSolver(case, "f64", ib=ib)
    gpu.set_macro(*init())
    gpu.step(3, record_force=True)
    r1 = gpu.compute_ib_force()
    gpu.have_prev_body = False
    r2 = gpu.compute_ib_force()
    np.testing.assert_array_equal(r1[9:12], r2[9:12])
    F = gpu.get_force()
    dV = case.dx ** 2
    np.testing.assert_allclose(r1[9:11], -F[:2].reshape(2, -1).sum(axis=1) * dV / case.dt, rtol=1e-12)
    gpu.close()


def test_bad_arguments_return_errors():
    from ilbmrex_b200.level import Context, level_params
    case, init = cases.taylor_green(16)
    ctx = Context(case.lattice, "f64")
    p = level_params(case, uniform_force=True)
    b = capi.Box_t()
    rc = ctx.L.ilbm_level_step(ctx.h, C.byref(b), 1, C.byref(p))
    assert rc != 0
    p.tau = 0.4
    rc = ctx.L.ilbm_level_step(ctx.h, C.byref(b), 1, C.byref(p))
    assert rc != 0 and b"tau" in ctx.L.ilbm_last_error()
    ctx.close()
