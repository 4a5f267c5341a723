"""ilbm_force_integrals_noalloc (no device allocation) against
ilbm_force_integrals, both through the C ABI.  Kept in its own file, collected
last, so it runs both alone in a fresh process and after the rest of the suite."""
import ctypes as C

import numpy as np
import pytest

from ilbmrex_b200 import capi, cases

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.level import Context, LevelSolver  # noqa: E402


def _sum(L, fn, ctx, box, force_ptr, lo, hi):
    """ilbm_force_integrals takes the force array in the box (a list of one
    box here); the no-allocation entry point takes one box and the array."""
    out = (C.c_double * 3)()
    if fn == "ilbm_force_integrals":
        b = capi.Box_t.from_buffer_copy(box)
        b.force = force_ptr
        rc = L.ilbm_force_integrals(ctx, C.byref(b), 1, capi.ivec3(lo), capi.ivec3(hi), out)
    else:
        rc = getattr(L, fn)(ctx, C.byref(box), force_ptr, capi.ivec3(lo), capi.ivec3(hi), out)
    return rc, np.array([out[0], out[1], out[2]])


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_noalloc_matches_force_integrals(storage):
    case, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    gpu = LevelSolver(case, storage, ib=ib)
    gpu.set_macro(*init())
    gpu.step(3)
    gpu.ctx.sync()
    L, h = gpu.L, gpu.ctx.h
    box = gpu._box(gpu.f, None)
    fptr = gpu.force_prev.data_ptr()
    lo, hi = gpu.force_region
    rc, ref = _sum(L, "ilbm_force_integrals", h, box, fptr, lo, hi)
    assert rc == 0
    assert np.abs(ref[:2]).max() > 0.0
    got = []
    for _ in range(2):  # two calls in a row: same bits, same sum as the existing entry point
        rc, s = _sum(L, "ilbm_force_integrals_noalloc", h, box, fptr, lo, hi)
        assert rc == 0, L.ilbm_last_error()
        got.append(s)
    np.testing.assert_array_equal(got[0], got[1])
    np.testing.assert_allclose(got[0], ref, rtol=1e-12, atol=1e-15)
    # whole box (region NULL -> the box)
    rc, ref_all = _sum(L, "ilbm_force_integrals", h, box, fptr, (0, 0, 0), (10**6, 10**6, 10**6))
    rc2, got_all = _sum(L, "ilbm_force_integrals_noalloc", h, box, fptr, (0, 0, 0), (10**6, 10**6, 10**6))
    assert rc == 0 and rc2 == 0
    np.testing.assert_allclose(got_all, ref_all, rtol=1e-12, atol=1e-15)
    gpu.close()


def test_noalloc_size_limit():
    """8,388,608 cells is the largest region; one more row is refused before
    anything is launched."""
    ctx = Context(cases.D2Q9, "f32")
    L = ctx.L
    nx, ny = 4096, 2049
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(20261203)
    F = torch.rand((3, ny, nx), generator=g, device=dev, dtype=torch.float32) - 0.5
    torch.cuda.synchronize()
    b = capi.Box_t()
    b.lo[0], b.lo[1], b.lo[2] = 0, 0, 0
    b.hi[0], b.hi[1], b.hi[2] = nx - 1, ny - 1, 0
    b.ngrow_f, b.ngrow_m = 0, 0
    b.mstride[0], b.mstride[1], b.mstride[2] = nx, nx * ny, nx * ny
    fptr = F.data_ptr()
    at_limit = ((0, 0, 0), (nx - 1, ny - 2, 0))  # 4096 x 2048 cells
    rc, ref = _sum(L, "ilbm_force_integrals", ctx.h, b, fptr, *at_limit)
    assert rc == 0
    for _ in range(2):
        rc, s = _sum(L, "ilbm_force_integrals_noalloc", ctx.h, b, fptr, *at_limit)
        assert rc == 0, L.ilbm_last_error()
        np.testing.assert_allclose(s, ref, rtol=1e-9, atol=1e-9)
    host = F[:, :ny - 1, :].double().sum(dim=(1, 2)).cpu().numpy()
    np.testing.assert_allclose(s[:2], host[:2], rtol=1e-9, atol=1e-6)
    rc, _ = _sum(L, "ilbm_force_integrals_noalloc", ctx.h, b, fptr, (0, 0, 0), (nx - 1, ny - 1, 0))
    assert rc == capi.ILBM_ERR_RANGE
    assert b"8388608" in L.ilbm_last_error()
    ctx.close()


def _offset_box(nx, ny, lo=(5, 7), ng=2, seed=20261203):
    """A 2D box whose valid region starts at `lo` (not the origin) inside a
    force array grown by `ng` ghost cells; the ghosts hold large values that a
    wrong offset would pick up."""
    dev = torch.device("cuda", 0)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    gx, gy = nx + 2 * ng, ny + 2 * ng
    F = torch.full((3, gy, gx), 1.0e6, device=dev, dtype=torch.float64)
    F[:, ng:ng + ny, ng:ng + nx] = torch.rand((3, ny, nx), generator=g, device=dev,
                                              dtype=torch.float64) - 0.5
    torch.cuda.synchronize()
    b = capi.Box_t()
    b.lo[0], b.lo[1], b.lo[2] = lo[0], lo[1], 0
    b.hi[0], b.hi[1], b.hi[2] = lo[0] + nx - 1, lo[1] + ny - 1, 0
    b.ngrow_f, b.ngrow_m = ng, ng
    b.mstride[0], b.mstride[1], b.mstride[2] = gx, gx * gy, gx * gy
    return F, b


def test_noalloc_offset_box_ragged_chunks():
    """A region of 241 x 32 = 7,712 cells (two chunks, the last one ragged) on
    a box whose lo is (5, 7) with two ghost layers: equal to
    ilbm_force_integrals and to a float64 sum of the same cells."""
    ctx = Context(cases.D2Q9, "f64")
    L = ctx.L
    nx, ny, lo = 300, 50, (5, 7)
    F, b = _offset_box(nx, ny, lo)
    rlo, rhi = (lo[0] + 10, lo[1] + 9, 0), (lo[0] + 250, lo[1] + 40, 0)
    rc, ref = _sum(L, "ilbm_force_integrals", ctx.h, b, F.data_ptr(), rlo, rhi)
    assert rc == 0
    ng = 2
    i0, i1 = rlo[0] - lo[0] + ng, rhi[0] - lo[0] + ng + 1
    j0, j1 = rlo[1] - lo[1] + ng, rhi[1] - lo[1] + ng + 1
    host = F[:, j0:j1, i0:i1].sum(dim=(1, 2)).cpu().numpy()
    for _ in range(2):
        rc, s = _sum(L, "ilbm_force_integrals_noalloc", ctx.h, b, F.data_ptr(), rlo, rhi)
        assert rc == 0, L.ilbm_last_error()
        np.testing.assert_allclose(s, ref, rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(s[:2], host[:2], rtol=1e-12, atol=1e-12)
    ctx.close()


def test_noalloc_empty_region():
    """A region that clips to nothing returns ILBM_OK and zeros, like
    ilbm_force_integrals, after a call that left a nonzero sum behind."""
    ctx = Context(cases.D2Q9, "f64")
    L = ctx.L
    F, b = _offset_box(64, 40)
    rc, s = _sum(L, "ilbm_force_integrals_noalloc", ctx.h, b, F.data_ptr(), (5, 7, 0), (68, 46, 0))
    assert rc == 0 and np.abs(s).max() > 0.0
    for rlo, rhi in (((200, 7, 0), (300, 46, 0)), ((30, 20, 0), (29, 30, 0))):
        rc, ref = _sum(L, "ilbm_force_integrals", ctx.h, b, F.data_ptr(), rlo, rhi)
        assert rc == 0
        rc, s = _sum(L, "ilbm_force_integrals_noalloc", ctx.h, b, F.data_ptr(), rlo, rhi)
        assert rc == 0, L.ilbm_last_error()
        np.testing.assert_array_equal(s, np.zeros(3))
        np.testing.assert_array_equal(ref, np.zeros(3))
    ctx.close()
