"""Derived fields (vorticity, pressure) and ErrorEst refinement tags through
the C ABI against the restated visPara / ErrorEst applied to the oracle's
own FillPatched macro fields.  FP64 storage: bit-exact without a body; with
an immersed body the marker forces are spread with FP64 atomics in no fixed
order, so the level's velocity (and everything after it) agrees to 1e-12 of
the field's largest value.  The tags are checked bit for bit against the
restated ErrorEst applied to the device's own vorticity."""
import numpy as np
import pytest

from ilbmrex_b200 import cases
from oracle.checker import CpuLevel, error_est_tags, vorticity_pressure

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.level import LevelSolver, refinement_region  # noqa: E402


def _pair(case, ib, init, steps):
    cpu = CpuLevel(case, "oracle")
    cpu.set_macro(*init())
    cpu.init_equilibrium()
    if ib is not None:
        cpu.ib_create(ib)
    cpu.step(steps)
    gpu = LevelSolver(case, "f64", ib=ib)
    gpu.set_macro(*init())
    gpu.step(steps)
    ng = case.nghost
    nx, ny, nz = case.n_cell
    gz = nz + 2 * ng if case.dim == 3 else 1
    mg = cpu.fill_patch_macro().reshape(6, gz, ny + 2 * ng, nx + 2 * ng)
    return cpu, gpu, mg


@pytest.mark.parametrize("which", ["cylinder2d", "channel2d", "sphere3d", "duct3d"])
def test_vorticity_pressure_and_tags(which):
    if which == "cylinder2d":
        case, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    elif which == "channel2d":
        (case, init), ib = cases.channel_bounce_back(nx=40, ny=24), None
    elif which == "sphere3d":
        case, ib, init = cases.sphere(48, 32, 32, D=12.0, center=(16.3, 15.8, 16.1), U=0.04, Re=40.0)
    else:
        (case, init), ib = cases.square_duct(N=10, L=6, force=1e-4, nu=0.06), None
    cpu, gpu, mg = _pair(case, ib, init, 5)
    vor, pres, vmax = gpu.derived_fields()
    vref, pref = vorticity_pressure(mg, case.nghost, case.dim, case.dx, case.dx, case.dx)
    if ib is None:
        np.testing.assert_array_equal(vor, vref)
        np.testing.assert_array_equal(pres, pref)
        assert vmax == vref.max()
    else:
        np.testing.assert_allclose(vor, vref, rtol=0, atol=1e-12 * np.abs(vref).max())
        np.testing.assert_allclose(pres, pref, rtol=0, atol=1e-12 * np.abs(pref).max())
        assert abs(vmax - vref.max()) <= 1e-12 * vref.max()
    assert vmax == vor.max()
    # the body box holds the whole level-set band, so the band alone is
    # tried with the box off
    for ratio, nr, use_box, use_ls in ((0.3, (0.0, 0.0), True, True),
                                       (0.05, (4.0, 6.0), True, True),
                                       (0.3, (0.0, 0.0), False, True),
                                       (0.3, (0.0, 0.0), True, False)):
        tags, n, thr = gpu.tag_cells(ratio, refine_box=use_box, no_refine=nr, levelset=use_ls)
        box = refinement_region(case, ib) if ib is not None and use_box else None
        ls = None
        if use_ls and ib is not None:
            ls = (ib.x0, ib.y0, ib.z0 if case.dim == 3 else 0.0, ib.R, 5, case.dx)
        assert thr == ratio * vmax
        ref = error_est_tags(vor, thr, case.prob_lo, case.prob_hi, [case.dx] * 3, box, nr, ls)
        np.testing.assert_array_equal(tags, ref)
        assert n == int(ref.sum())
        assert n > 0 or nr != (0.0, 0.0)
    gpu.close()
