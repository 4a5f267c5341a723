"""Static two-level hierarchy on the GPU (ilbm_advance_two_level) against the
oracle's two-level driver (oracle/lbm_oracle.c, orc2_*), same seeded fields.

FP64 storage without a body: both levels' populations and stored macro
fields bit for bit (the coarse-fine fill, the subcycled steps and the
average-down keep the oracle's operation order).  With a body on the fine
level the marker forces are spread with FP64 atomics: relative L2 <= 1e-12
and force coefficients to 1e-9.  FP32 / FP16 storage: the velocity fields
within the bounds of the single-level storage tests.
"""
import numpy as np
import pytest

from ilbmrex_b200 import cases
from oracle.checker import CpuTwoLevel

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.hierarchy import TwoLevelSolver  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def _pair(tl, ic, if_, ib, storage, steps):
    cpu = CpuTwoLevel(tl)
    cpu.set_macro(0, *ic())
    cpu.set_macro(1, *if_())
    cpu.init_equilibrium()
    if ib is not None:
        cpu.ib_create(ib)
    gpu = TwoLevelSolver(tl, storage, ib=ib)
    gpu.set_macro(ic(), if_())
    for lev in (0, 1):
        if storage == "f64":
            np.testing.assert_array_equal(gpu.get_f(lev), cpu.get_f(lev))
    cpu.step(steps)
    gpu.step(steps, record_force=ib is not None)
    return cpu, gpu


@pytest.mark.parametrize("lattice", ["d2q9", "d3q19"])
def test_shear_layer_bit_exact(lattice):
    if lattice == "d2q9":
        tl, ic, if_ = cases.shear_layer_two_level(n=48, fine=(24, 72))
        steps = 12
    else:
        tl, ic, if_ = cases.shear_layer_two_level(n=20, fine=(12, 28), lattice=cases.D3Q19)
        steps = 5
    cpu, gpu = _pair(tl, ic, if_, None, "f64", steps)
    for lev in (0, 1):
        np.testing.assert_array_equal(gpu.get_f(lev), cpu.get_f(lev))
        np.testing.assert_array_equal(gpu.get_macro(lev), cpu.get_macro(lev))
    # the fine level carries structure the coarse one does not resolve alone
    assert np.abs(gpu.get_macro(1)[1]).max() > 0.0
    gpu.close()


def test_cylinder_body_on_fine_level():
    tl, ib, ic, if_ = cases.cylinder_two_level(nx=96, ny=64, D=12.0, center=(32.3, 31.7), U=0.05,
                                               Re=40.0, upstream=1.0, downstream=2.0, cross=1.2)
    cpu, gpu = _pair(tl, ic, if_, ib, "f64", 6)
    for lev in (0, 1):
        assert rel_l2(gpu.get_f(lev), cpu.get_f(lev)) <= 1e-12
    np.testing.assert_allclose(gpu.rec[3:5], cpu.force_record()[3:5], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(gpu.marker_force_sum(), cpu.marker_force_sum(), rtol=1e-9, atol=1e-14)
    gpu.close()


@pytest.mark.parametrize("storage,tol", [("f32", 2e-5), ("f16", 5e-3)])
def test_shear_layer_storage_forms(storage, tol):
    tl, ic, if_ = cases.shear_layer_two_level(n=48, fine=(24, 72))
    cpu, gpu = _pair(tl, ic, if_, None, storage, 12)
    for lev in (0, 1):
        g, c = gpu.get_macro(lev), cpu.get_macro(lev)
        scale = np.abs(c[1:3]).max()  # the flow's velocity scale
        for n in (1, 2):
            assert np.abs(g[n] - c[n]).max() <= tol * scale, (lev, n)
    gpu.close()


def test_uniform_flow_stays_uniform():
    """A uniform state is a fixed point of the coarse-fine fill, the
    subcycling and the average-down."""
    c = cases.LevelCase(cases.D2Q9, (32, 32, 1), nu=0.02)
    tl = cases.TwoLevelCase(c, (16, 16), (47, 47))
    ic = cases.uniform_init(c, 1.0, (0.03, -0.01, 0.0))
    if_ = cases.uniform_init(tl.fine_box(), 1.0, (0.03, -0.01, 0.0))
    gpu = TwoLevelSolver(tl, "f64")
    gpu.set_macro(ic(), if_())
    gpu.step(6)
    for lev in (0, 1):
        m = gpu.get_macro(lev)
        assert np.abs(m[1] - 0.03).max() < 1e-14 and np.abs(m[2] + 0.01).max() < 1e-14
        assert np.abs(m[0] - 1.0).max() < 1e-14
    gpu.close()


def test_sphere_body_on_fine_level_3d():
    """The headline's machinery at test size: D3Q19, two levels, a sphere on
    the fine level with more than 1024 markers (grid CG, extrapolated starts),
    its forcing overlapped with the level steps; FP64 against the oracle's
    two-level driver with dense LU (relative L2 <= 1e-12)."""
    tl, ib, ic, if_ = cases.sphere_two_level(nx=32, ny=24, nz=24, D=10.0, center=(12.3, 11.8, 12.1),
                                             U=0.04, Re=30.0, box_lo=(4, 4, 4), box_hi=(22, 20, 20))
    cpu, gpu = _pair(tl, ic, if_, ib, "f64", 4)
    n = __import__("ctypes").c_int64()
    gpu.L.ilbm_ib_num_markers(gpu.ib, __import__("ctypes").byref(n))
    assert n.value > 1024
    for lev in (0, 1):
        assert rel_l2(gpu.get_f(lev), cpu.get_f(lev)) <= 1e-12
        assert rel_l2(gpu.get_macro(lev), cpu.get_macro(lev)) <= 1e-12
    np.testing.assert_allclose(gpu.rec[3:5], cpu.force_record()[3:5], rtol=1e-9, atol=1e-12)
    gpu.close()


def test_pipelined_force_records():
    """ilbm_force_record_async: with pipelined records each step's record is
    taken once the next step is queued (one step behind during the loop,
    flush_records takes the last) and equals the synchronous record."""
    tl, ib, ic, if_ = cases.cylinder_two_level(nx=96, ny=64, D=12.0, center=(32.3, 31.7), U=0.05,
                                               Re=40.0, upstream=1.0, downstream=2.0, cross=1.2)
    a = TwoLevelSolver(tl, "f64", ib=ib)
    b = TwoLevelSolver(tl, "f64", ib=ib)
    for s in (a, b):
        s.set_macro(ic(), if_())
    recs = []
    for k in range(5):
        a.advance(record_force=True)
        recs.append(a.rec.copy())
        b.advance(record_force=True, pipelined=True)
        if k >= 1:
            np.testing.assert_allclose(b.rec, recs[k - 1], rtol=1e-9, atol=1e-14)
    b.flush_records()
    np.testing.assert_allclose(b.rec, recs[-1], rtol=1e-9, atol=1e-14)
    assert abs(recs[-1][3]) > 0.0
    a.close()
    b.close()


def test_force_record_into_pageable_pinned_and_device_memory():
    """ilbm_force_record_async writes pinned host and device buffers from its
    last kernel and copies into pageable memory: the three records are the
    same bits, and equal ilbm_force_integrals and the last marker force sum
    (the same fixed-order reduction)."""
    import ctypes as C
    from ilbmrex_b200 import capi
    tl, ib, ic, if_ = cases.cylinder_two_level(nx=96, ny=64, D=12.0, center=(32.3, 31.7), U=0.05,
                                               Re=40.0, upstream=1.0, downstream=2.0, cross=1.2)
    s = TwoLevelSolver(tl, "f64", ib=ib)
    s.set_macro(ic(), if_())
    s.step(3)
    lo, hi = s.force_region
    b = s.F.box(s.F.f, None, force=s.F.fb)
    page = np.full(8, np.nan)
    pin = torch.full((8,), float("nan"), dtype=torch.float64).pin_memory()
    dev = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")
    for ptr in (page.ctypes.data, pin.data_ptr(), dev.data_ptr()):
        capi.check(s.L.ilbm_force_record_async(s.ctx.h, C.byref(b), 1, s.ib, capi.ivec3(lo),
                                               capi.ivec3(hi), C.c_void_p(ptr)), "force_record_async")
    s.ctx.sync()
    np.testing.assert_array_equal(pin.numpy(), page)
    np.testing.assert_array_equal(dev.cpu().numpy(), page)
    e = (C.c_double * 3)()
    capi.check(s.L.ilbm_force_integrals(s.ctx.h, C.byref(b), 1, capi.ivec3(lo), capi.ivec3(hi), e),
               "force_integrals")
    m = (C.c_double * 3)()
    capi.check(s.L.ilbm_ib_last_marker_force_sum(s.ib, m), "marker_force_sum")
    np.testing.assert_array_equal(page[:3], np.array(e[:]))
    np.testing.assert_array_equal(page[3:6], np.array(m[:]))
    assert page[6] == 0.0 and page[7] == 0.0  # status words
    assert abs(page[0]) > 0.0
    s.close()


def test_step_with_record_into_pageable_memory():
    """ilbm_advance_two_level_recorded with a pageable buffer takes the step,
    then ilbm_force_record_async: the record equals the force integrals and
    the marker force sum of the step (the pinned-buffer form, whose record
    runs beside the step's end, is what test_pipelined_force_records uses)."""
    import ctypes as C
    from ilbmrex_b200 import capi

    class _Host:
        def __init__(self, a):
            self.a = a

        def data_ptr(self):
            return self.a.ctypes.data

    tl, ib, ic, if_ = cases.cylinder_two_level(nx=96, ny=64, D=12.0, center=(32.3, 31.7), U=0.05,
                                               Re=40.0, upstream=1.0, downstream=2.0, cross=1.2)
    s = TwoLevelSolver(tl, "f64", ib=ib)
    s.set_macro(ic(), if_())
    s.step(2)
    page = np.full(8, np.nan)
    s._launch_step(record_into=_Host(page))
    Cl = s.C
    Cl.f, Cl.f_next = Cl.f_next, Cl.f
    Cl.m, Cl.m_next = Cl.m_next, Cl.m
    s.time += s.hc.coarse.dt
    s.ctx.sync()
    lo, hi = s.force_region
    b = s.F.box(s.F.f, None, force=s.F.fb)
    e = (C.c_double * 3)()
    capi.check(s.L.ilbm_force_integrals(s.ctx.h, C.byref(b), 1, capi.ivec3(lo), capi.ivec3(hi), e),
               "force_integrals")
    m = (C.c_double * 3)()
    capi.check(s.L.ilbm_ib_last_marker_force_sum(s.ib, m), "marker_force_sum")
    np.testing.assert_array_equal(page[:3], np.array(e[:]))
    np.testing.assert_array_equal(page[3:6], np.array(m[:]))
    assert page[6] == 0.0 and page[7] == 0.0 and abs(page[0]) > 0.0
    s.close()
