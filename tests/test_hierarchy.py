"""Static hierarchies deeper than two levels (ilbm_advance_hierarchy) against
the oracle's N-level driver (orcN_*, restating timeStepWithSubcycling's
recursion, Source/Core/AmrCoreLBM.cpp:1690-1755).

* without a body, FP64: bit-exact on every level;
* with the marker IBM on the finest level, FP64: relative L2 <= 1e-12 on every
  level (the IVC system is solved through the stored inverse or CG instead of
  the reference's dense LU, and spreading sums in atomic order), Cd / Cl
  rtol 1e-9;
* two levels through ilbm_advance_hierarchy equal ilbm_advance_two_level;
* the cylinder of the benchmark's two-AMR-level configuration (1024 x 512 base
  level, max_level 2) against the oracle at full size, Cd / Cl within 0.1%.
"""
import numpy as np
import pytest

from ilbmrex_b200 import cases
from oracle.checker import CpuHierarchy, CpuTwoLevel

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.hierarchy import HierarchySolver, TwoLevelSolver  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def _pair(hc, inits, ib, storage, steps, record=False):
    cpu = CpuHierarchy(hc)
    for l, init in enumerate(inits):
        cpu.set_macro(l, *init())
    cpu.init_equilibrium()
    if ib is not None:
        cpu.ib_create(ib)
    cpu.step(steps)
    gpu = HierarchySolver(hc, storage, ib=ib)
    gpu.set_macro([init() for init in inits])
    if record and ib is not None:
        gpu.step(steps - 2)
        gpu.step(2, record_force=True)
    else:
        gpu.step(steps)
    return cpu, gpu


@pytest.mark.parametrize("lattice,n", [(cases.D2Q9, 64), (cases.D3Q19, 32)])
def test_three_levels_without_body_bit_exact(lattice, n):
    hc, inits = cases.shear_layer_hierarchy(n, nlev=3, lattice=lattice)
    cpu, gpu = _pair(hc, inits, None, "f64", 5)
    for lev in range(3):
        np.testing.assert_array_equal(gpu.get_f(lev), cpu.get_f(lev))
        np.testing.assert_array_equal(gpu.get_macro(lev), cpu.get_macro(lev))
    gpu.close()


def test_four_levels_without_body_bit_exact():
    hc, inits = cases.shear_layer_hierarchy(64, nlev=4)
    cpu, gpu = _pair(hc, inits, None, "f64", 3)
    for lev in range(4):
        np.testing.assert_array_equal(gpu.get_f(lev), cpu.get_f(lev))
    gpu.close()


def test_three_levels_cylinder_on_finest():
    hc, ib, inits = cases.cylinder_hierarchy(nx=128, ny=96, D=12.0, center=(40.3, 47.6), U=0.05, Re=40.0,
                                             nlev=3, upstream=0.8, downstream=1.6, cross=1.0, grow=6)
    cpu, gpu = _pair(hc, inits, ib, "f64", 6, record=True)
    for lev in range(3):
        assert rel_l2(gpu.get_f(lev), cpu.get_f(lev)) <= 1e-12, lev
        mg, mc = gpu.get_macro(lev), cpu.get_macro(lev)
        assert rel_l2(mg[0], mc[0]) <= 1e-12, lev
        assert rel_l2(mg[1:3], mc[1:3]) <= 1e-12, lev
    rg, rc = gpu.rec, cpu.force_record()
    np.testing.assert_allclose(rg[3], rc[3], rtol=1e-9)
    assert abs(rg[4] - rc[4]) <= 1e-9 * abs(rc[3])
    gpu.close()


def test_two_levels_through_the_hierarchy_call():
    """ilbm_advance_hierarchy with two levels gives ilbm_advance_two_level's
    result: bit for bit without a body, <= 1e-12 with one (the two schedules
    interleave the body's forcing differently: atomic spreading order)."""
    tl, ib, ic, if_ = cases.cylinder_two_level(nx=96, ny=64, D=12.0, center=(32.3, 31.7), U=0.05,
                                               Re=40.0, upstream=1.0, downstream=2.0, cross=1.2)
    hc = cases.HierarchyCase(tl.coarse, ((tl.fine_lo, tl.fine_hi),))
    for body in (None, ib):
        a = TwoLevelSolver(tl, "f64", ib=body)
        b = HierarchySolver(hc, "f64", ib=body)
        a.set_macro(ic(), if_())
        b.set_macro(ic(), if_())
        a.step(4)
        b.step(4)
        for lev in (0, 1):
            if body is None:
                np.testing.assert_array_equal(a.get_f(lev), b.get_f(lev))
            else:
                assert rel_l2(a.get_f(lev), b.get_f(lev)) <= 1e-12
        a.close()
        b.close()
    # and the oracle's two-level driver is the N-level one with two levels
    cpu = CpuTwoLevel(tl)
    cpu.set_macro(0, *ic())
    cpu.set_macro(1, *if_())
    cpu.init_equilibrium()
    cpu.step(3)
    g = TwoLevelSolver(tl, "f64")
    g.set_macro(ic(), if_())
    g.step(3)
    for lev in (0, 1):
        np.testing.assert_array_equal(g.get_f(lev), cpu.get_f(lev))
    g.close()


def _cylinder_three_levels():
    """The benchmark's cylinder with two refined levels (max_level 2): base
    1024 x 512, D = 40 at (256, 256), U = 0.05, Re = 100; the finest box 1 R
    upstream, 4 R downstream and 2 R across plus 6 base cells, the middle
    level around it."""
    R, pad = 20.0, 6.0
    return cases.cylinder_hierarchy(nx=1024, ny=512, D=2 * R, center=(256.0, 256.0), U=0.05, Re=100.0,
                                    nlev=3, upstream=(R + pad) / (2 * R), downstream=(4 * R + pad) / (2 * R),
                                    cross=(2 * R + pad) / (2 * R))


def test_cylinder_1024x512_three_levels_fp64():
    hc, ib, inits = _cylinder_three_levels()
    cpu, gpu = _pair(hc, inits, ib, "f64", 60, record=True)
    for lev in range(3):
        assert rel_l2(gpu.get_f(lev), cpu.get_f(lev)) <= 1e-12, lev
    rg, rc = gpu.rec, cpu.force_record()
    assert abs(rg[3] - rc[3]) <= 1e-3 * abs(rc[3])
    assert abs(rg[4] - rc[4]) <= 1e-3 * abs(rc[3])
    gpu.close()
