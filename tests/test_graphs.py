"""Hierarchy steps replayed from a CUDA graph (``graphs=True``: two coarse
steps recorded once through ``ilbm_graph_begin`` / ``ilbm_graph_end`` and
replayed by ``ilbm_graph_launch``) against the same steps issued one call at
a time:

* the three-level cylinder (stored IVC inverse) and the two-level sphere (the
  grid-wide CG, its solver history kept on the device) in FP64: bit for bit,
  with the same number of kernel launches;
* the three-level cylinder in FP32, whose spreading adds atomically: within
  FP32 rounding.
"""
import ctypes as C

import numpy as np
import pytest

from ilbmrex_b200 import capi, cases

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.hierarchy import HierarchySolver, TwoLevelSolver  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def _cylinder():
    hc, ib, inits = cases.cylinder_hierarchy(nx=128, ny=96, D=12.0, center=(40.3, 47.6), U=0.05, Re=40.0,
                                             nlev=3, upstream=0.8, downstream=1.6, cross=1.0, grow=6)
    return lambda g, st: HierarchySolver(hc, st, ib=ib, graphs=g), [init() for init in inits]


def _sphere():
    tl, ib, ic, if_ = cases.sphere_two_level(nx=32, ny=24, nz=24, D=10.0, center=(12.3, 11.8, 12.1),
                                             U=0.04, Re=30.0, box_lo=(4, 4, 4), box_hi=(22, 20, 20))
    return lambda g, st: TwoLevelSolver(tl, st, ib=ib, graphs=g), [ic(), if_()]


def _run(make, storage, graphs, steps, solver=None):
    new, inits = make()
    s = new(graphs, storage)
    if solver is not None:
        capi.check(s.L.ilbm_ib_set_ivc_solver(s.ib, solver), "set_ivc_solver")
    s.set_macro(*inits)
    s.step(1)  # the first step (tables, stored macro fields) as one call
    l0 = s.ctx.launches()
    s.step(steps)
    launches = s.ctx.launches() - l0
    s.step(2, record_force=True)
    out = ([s.get_f(l) for l in range(s.nlev)], s.rec.copy(), launches, s._graph is not None)
    s.close()
    return out


@pytest.mark.parametrize("make,solver", [(_cylinder, None), (_sphere, capi.IVC_CG)],
                         ids=["cylinder_3lev", "sphere_2lev_cg"])
def test_graph_replay_equals_calls_fp64(make, solver):
    fa, ra, la, ga = _run(make, "f64", False, 8, solver)
    fb, rb, lb, gb = _run(make, "f64", True, 8, solver)
    assert not ga and gb
    for lev, (x, y) in enumerate(zip(fa, fb)):
        assert np.array_equal(x, y), lev
    assert np.array_equal(ra, rb)
    assert la == lb


def test_graph_replay_fp32_cylinder():
    fa, ra, _, _ = _run(_cylinder, "f32", False, 8)
    fb, rb, _, gb = _run(_cylinder, "f32", True, 8)
    assert gb
    for lev, (x, y) in enumerate(zip(fa, fb)):
        assert rel_l2(y, x) <= 1e-6, lev
    np.testing.assert_allclose(rb[3:5], ra[3:5], rtol=1e-5, atol=1e-9)
