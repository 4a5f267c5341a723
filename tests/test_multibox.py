"""A level held in several boxes with caller-filled ghosts (the AMReX drop-in
mode, a level cut by max_grid_size): the marker IBM, the level step, the force
integral and the momentum exchange through the C ABI against the oracle's
single-box run of the same step.

The caller's FillPatch is the oracle's (fill_patch_f / fill_patch_macro of
the state after N steps); each box gets its valid cells plus one ghost layer
of f^n and two of rho, u.  After ilbm_ib_update_forcing on all boxes and
ilbm_level_step on all boxes, the stitched populations and forces must equal
the oracle's step N+1: relative L2 <= 1e-12 (force field 1e-11).
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

from ilbmrex_b200.level import Context, LevelSolver, ib_params, level_geom, level_params  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


class Boxes:
    """Device arrays of the boxes of one 2D level (f grown by 1, macro and
    force grown by 2), filled from the oracle's FillPatched grown arrays."""

    def __init__(self, case, fg, mg, cuts_x, cuts_y, ng):
        self.case, self.ng = case, ng
        nx, ny = case.n_cell[0], case.n_cell[1]
        xs = [0] + list(cuts_x) + [nx]
        ys = [0] + list(cuts_y) + [ny]
        self.ranges = [((xs[a], xs[a + 1] - 1), (ys[b], ys[b + 1] - 1))
                       for b in range(len(ys) - 1) for a in range(len(xs) - 1)]
        dev = torch.device("cuda", 0)
        self.keep = []
        self.arr = (capi.Box_t * len(self.ranges))()
        lb = []
        for n, ((i0, i1), (j0, j1)) in enumerate(self.ranges):
            w, h = i1 - i0 + 1, j1 - j0 + 1
            fin = torch.tensor(fg[:, j0 - 1 + ng:j1 + 2 + ng, i0 - 1 + ng:i1 + 2 + ng],
                               dtype=torch.float64, device=dev).contiguous()
            mac = torch.tensor(mg[:4, j0 - 2 + ng:j1 + 3 + ng, i0 - 2 + ng:i1 + 3 + ng],
                               dtype=torch.float64, device=dev).contiguous()
            fout = torch.zeros_like(fin)
            force = torch.zeros((3, h + 4, w + 4), dtype=torch.float64, device=dev)
            self.keep.append((fin, fout, mac, force))
            B = self.arr[n]
            B.lo[0], B.lo[1], B.lo[2] = i0, j0, 0
            B.hi[0], B.hi[1], B.hi[2] = i1, j1, 0
            B.ngrow_f, B.ngrow_m = 1, 2
            B.fstride[0], B.fstride[1], B.fstride[2] = w + 2, (w + 2) * (h + 2), (w + 2) * (h + 2)
            B.mstride[0], B.mstride[1], B.mstride[2] = w + 4, (w + 4) * (h + 4), (w + 4) * (h + 4)
            B.f_in, B.f_out = fin.data_ptr(), fout.data_ptr()
            B.macro_in, B.force = mac.data_ptr(), force.data_ptr()
            lb += [i0, j0, 0, i1, j1, 0]
        self.lb = (C.c_int * len(lb))(*lb)
        torch.cuda.synchronize()

    def stitch(self, which):
        """Valid cells of f_out (which = 1, [Q, 1, ny, nx]) or of the force
        (which = 3, [3, 1, ny, nx]) over the level."""
        nx, ny = self.case.n_cell[0], self.case.n_cell[1]
        comps = self.case.lattice.q if which == 1 else 3
        out = np.zeros((comps, 1, ny, nx))
        for ((i0, i1), (j0, j1)), t in zip(self.ranges, self.keep):
            g = 1 if which == 1 else 2
            a = t[which].cpu().numpy()
            out[:, 0, j0:j1 + 1, i0:i1 + 1] = a[:comps, g:g + j1 - j0 + 1, g:g + i1 - i0 + 1]
        return out


def _two_ways(name, cuts_x, cuts_y, steps=3):
    builder, _ = GOLDEN_CASES[name]
    case, init, ib = builder()
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    cpu.ib_create(ib)
    cpu.step(steps)
    t = cpu.time
    ng = case.nghost
    nx, ny = case.n_cell[0], case.n_cell[1]
    fg = cpu.fill_patch_f().reshape(case.lattice.q, ny + 2 * ng, nx + 2 * ng)
    mg = cpu.fill_patch_macro().reshape(6, ny + 2 * ng, nx + 2 * ng)
    cpu.step(1)
    ctx = Context(case.lattice, "f64")
    L = ctx.L
    bx = Boxes(case, fg, mg, cuts_x, cuts_y, ng)
    p = level_params(case, uniform_force=False)
    p.ghost_mode = capi.GHOST_CALLER
    p.level_boxes = C.cast(bx.lb, C.POINTER(C.c_int))
    p.nlevel_boxes = len(bx.ranges)
    geom, ibp = level_geom(case), ib_params(ib, case.dim)
    h = C.c_void_p()
    capi.check(L.ilbm_ib_create(ctx.h, C.byref(ibp), C.byref(geom), C.byref(h)), "ib_create")
    lo, hi = (C.c_int * 3)(), (C.c_int * 3)()
    capi.check(L.ilbm_ib_force_region(h, lo, hi), "force_region")
    for d in range(3):
        p.force_lo[d], p.force_hi[d] = lo[d], hi[d]
    nb = len(bx.ranges)
    capi.check(L.ilbm_ib_update_forcing(h, bx.arr, nb, C.byref(p), case.dt, t), "update_forcing")
    capi.check(L.ilbm_level_step(ctx.h, bx.arr, nb, C.byref(p)), "level_step")
    ctx.sync()
    return cpu, ctx, h, bx, p, (tuple(lo), tuple(hi))


@pytest.mark.parametrize("name,cuts_x,cuts_y", [
    ("cylinder96x64_ivc", (32,), ()),                      # two boxes, the cut through the body
    ("cylinder96x64_ivc", (32,), (32,)),                   # four boxes meeting inside the body
    ("cylinder96x64_explicit_mdf2", (24, 40), (20, 44)),   # nine boxes, two MDF iterations
    ("cavity32_lid_box", (16,), (16,)),                    # lid markers along box faces
])
def test_ib_on_several_boxes_matches_oracle(name, cuts_x, cuts_y):
    cpu, ctx, ib, bx, p, _ = _two_ways(name, cuts_x, cuts_y)
    f, F = bx.stitch(1), bx.stitch(3)
    assert rel_l2(f, cpu.get_f()) <= 1e-12
    Fc = cpu.get_force()
    assert rel_l2(F[:2], Fc[:2]) <= 1e-11
    ctx.L.ilbm_ib_destroy(ib)
    ctx.close()


def test_force_integral_and_momentum_exchange_on_several_boxes():
    """The force integral over four boxes equals the one-box sum of the same
    field, and the momentum exchange over four boxes equals the one-box
    exchange (relative 1e-12: the summation is grouped by box)."""
    cpu, ctx, ib, bx, p, (flo, fhi) = _two_ways("cylinder96x64_ivc", (32,), (32,))
    L = ctx.L
    out4 = (C.c_double * 3)()
    capi.check(L.ilbm_force_integrals(ctx.h, bx.arr, len(bx.ranges), capi.ivec3(flo), capi.ivec3(fhi),
                                      out4), "integrals")
    F = torch.tensor(bx.stitch(3)[:, 0], dtype=torch.float64, device="cuda")
    ny, nx = F.shape[1], F.shape[2]
    one = capi.Box_t()
    one.lo[0], one.lo[1], one.lo[2] = 0, 0, 0
    one.hi[0], one.hi[1], one.hi[2] = nx - 1, ny - 1, 0
    one.ngrow_f, one.ngrow_m = 0, 0
    one.mstride[0], one.mstride[1], one.mstride[2] = nx, nx * ny, nx * ny
    one.force = F.data_ptr()
    out1 = (C.c_double * 3)()
    torch.cuda.synchronize()
    capi.check(L.ilbm_force_integrals(ctx.h, C.byref(one), 1, capi.ivec3(flo), capi.ivec3(fhi), out1),
               "integrals")
    np.testing.assert_allclose(list(out4)[:2], list(out1)[:2], rtol=1e-12, atol=1e-18)
    assert abs(out1[0]) > 0.0
    # momentum exchange of f^{n+1}: the stitched level as one box against the
    # four boxes (each one filled ghost layer: its neighbours' values)
    case = cpu.spec
    fl = bx.stitch(1)[:, 0]
    ng = 1
    fgrown = np.zeros((case.lattice.q, ny + 2 * ng, nx + 2 * ng))
    fgrown[:, ng:ng + ny, ng:ng + nx] = fl
    fone = torch.tensor(fgrown, dtype=torch.float64, device="cuda")
    one.ngrow_f = ng
    one.fstride[0], one.fstride[1], one.fstride[2] = nx + 2, (nx + 2) * (ny + 2), (nx + 2) * (ny + 2)
    one.f_in = fone.data_ptr()
    for n, ((i0, i1), (j0, j1)) in enumerate(bx.ranges):
        fin = bx.keep[n][0]
        fin.copy_(torch.tensor(fgrown[:, j0 - 1 + ng:j1 + 2 + ng, i0 - 1 + ng:i1 + 2 + ng], device="cuda"))
    torch.cuda.synchronize()
    x0, y0, R = 32.3, 31.7, 8.0
    dx = capi.dvec3([1.0] * 3)
    for one_sided in (0, 1):
        m1, m4 = (C.c_double * 3)(), (C.c_double * 3)()
        capi.check(L.ilbm_momentum_exchange(ctx.h, C.byref(one), 1, C.byref(p), x0, y0, 0.0, R,
                                            capi.dvec3(case.prob_lo), dx, one_sided, m1), "me1")
        capi.check(L.ilbm_momentum_exchange(ctx.h, bx.arr, len(bx.ranges), C.byref(p), x0, y0, 0.0, R,
                                            capi.dvec3(case.prob_lo), dx, one_sided, m4), "me4")
        np.testing.assert_allclose(list(m4)[:2], list(m1)[:2], rtol=1e-12, atol=1e-15)
        assert abs(m1[0]) > 0.0
    L.ilbm_ib_destroy(ib)
    ctx.close()


def test_several_boxes_need_caller_ghosts():
    """A level that is not one box holding the band is refused in self-fill
    mode (its ghosts would have to come from the caller)."""
    case, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    gpu = LevelSolver(case, "f64", ib=ib)
    gpu.set_macro(*init())
    b = gpu._box(gpu.f, gpu.f_next, macro_in=gpu.macro, force=gpu.force_cur)
    two = (capi.Box_t * 2)(b, b)
    two[0].hi[0] = 47
    two[1].lo[0] = 48
    rc = gpu.L.ilbm_ib_update_forcing(gpu.ib, two, 2, C.byref(gpu.params), case.dt, 0.0)
    assert rc == capi.ILBM_ERR_ARG and b"caller-filled" in gpu.L.ilbm_last_error()
    gpu.close()
