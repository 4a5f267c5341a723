"""Batch engine: every case advanced in the batch equals the same case
advanced alone through ilbm_advance_level (the single-case path, itself
checked against the oracle).  Differences come only from the order of the
FP64 atomics in force spreading: relative L2 <= 1e-12 with FP64 storage,
<= 1e-5 with FP32 storage (a force value may round to a neighbouring float)."""
import numpy as np
import pytest

from ilbmrex_b200 import cases
from ilbmrex_b200.lattice import D2Q9

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.batch import Batch  # noqa: E402
from ilbmrex_b200.level import LevelSolver  # noqa: E402

TOL = {"f64": (1e-12, 1e-9), "f32": (1e-5, 1e-4)}


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def mixed_cases():
    """(case, ib, init) of a small mixed D2Q9 set: two fixed cylinders (stored
    IVC inverse), a pitching airfoil (CG, operator rebuilt each step), a
    bounce-back channel and a periodic Taylor-Green box (no body)."""
    out = []
    out.append(cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40))
    out.append(cases.cylinder(nx=80, ny=48, D=12, center=(24.6, 23.2), U=0.04, Re=60))
    out.append(cases.pitching_airfoil(nx=128, ny=96, chord=32.0, pivot=(40.0, 48.0), U=0.05,
                                      Re=80.0, amplitude_deg=8.0, reduced_frequency=0.2))
    c, init = cases.channel_bounce_back(nx=40, ny=24)
    out.append((c, None, init))
    c, init = cases.taylor_green(48, U0=0.02, tau=0.7)
    out.append((c, None, init))
    return out


def alone(case, ib, init, storage, steps):
    s = LevelSolver(case, storage, ib=ib)
    s.set_macro(*init())
    s.step(steps, record_force=ib is not None)
    return s


@pytest.mark.parametrize("storage", ["f64", "f32"])
def test_batch_matches_cases_alone(storage):
    tf, tc = TOL[storage]
    n = 7  # an odd count: graph replays plus one direct step
    B = Batch(D2Q9, storage)
    ids = []
    for case, ib, init in mixed_cases():
        s = B.solver(case, ib, init)
        ids.append(B.add(s, max_steps=64))
    ncase, cells = B.size()
    assert ncase == 5 and cells > 0
    B.step(n)
    for cid, (case, ib, init) in zip(ids, mixed_cases()):
        s = B.sync(cid)
        assert s.istep == 1 + n
        ref = alone(case, ib, init, storage, 1 + n)
        assert rel_l2(s.get_f(), ref.get_f()) <= tf, case.name
        if ib is not None:
            np.testing.assert_allclose(s.rec[3:5], ref.rec[3:5], rtol=tc, atol=1e-12)
        assert abs(s.time - ref.time) == 0.0
        ref.close()
    B.close()


def test_batch_join_and_leave():
    """A case joins a running batch, another leaves it; both still match
    their runs alone."""
    storage = "f64"
    (ca, ia, xa), (cb, ib_, xb) = mixed_cases()[0], mixed_cases()[2]
    B = Batch(D2Q9, storage)
    sa = B.solver(ca, ia, xa)
    ida = B.add(sa, max_steps=64)
    B.step(4)
    sb = B.solver(cb, ib_, xb)
    idb = B.add(sb, max_steps=64)
    B.step(6)
    sa = B.remove(ida)
    assert sa.istep == 11
    ref = alone(ca, ia, xa, storage, 11)
    assert rel_l2(sa.get_f(), ref.get_f()) <= 1e-12
    np.testing.assert_allclose(sa.rec[3:5], ref.rec[3:5], rtol=1e-9, atol=1e-12)
    # the solver carries on alone from where the batch left it
    sa.step(3, record_force=True)
    ref.step(3, record_force=True)
    assert rel_l2(sa.get_f(), ref.get_f()) <= 1e-12
    B.step(3)
    sb = B.sync(idb)
    refb = alone(cb, ib_, xb, storage, 10)
    assert rel_l2(sb.get_f(), refb.get_f()) <= 1e-12
    sa.close()
    ref.close()
    refb.close()
    B.close()


def test_batch_tune_keeps_results():
    """The tuner's trial steps are real steps: the cases stay in step with
    their runs alone whatever tiling it picks."""
    storage = "f32"
    sel = [mixed_cases()[i] for i in (0, 3)]
    B = Batch(D2Q9, storage)
    ids = [B.add(B.solver(c, ib, x), max_steps=400) for c, ib, x in sel]
    w, cps, ms = B.tune(trial_steps=4)
    assert w in (64, 128, 256) and cps >= 1 and ms > 0.0
    B.step(5)
    for cid, (c, ib, x) in zip(ids, sel):
        s = B.sync(cid)
        ref = alone(c, ib, x, storage, s.istep)
        assert rel_l2(s.get_f(), ref.get_f()) <= 1e-5
        ref.close()
    B.close()


def test_case_stops_at_its_step_count():
    """A case added for 3 steps stops there on the device while the batch
    runs on; its state equals 1 + 3 steps alone, the other case's 1 + 9."""
    storage = "f64"
    (ca, ia, xa), (cb, ib_, xb) = mixed_cases()[1], mixed_cases()[2]
    B = Batch(D2Q9, storage)
    ida = B.add(B.solver(ca, ia, xa), max_steps=3)
    idb = B.add(B.solver(cb, ib_, xb), max_steps=100)
    B.step(9)
    prog = B.progress()
    assert prog[ida] == (3, 0) and prog[idb] == (9, 91)
    sa, sb = B.sync(ida), B.sync(idb)
    assert sa.istep == 4 and sb.istep == 10
    ra, rb = alone(ca, ia, xa, storage, 4), alone(cb, ib_, xb, storage, 10)
    assert rel_l2(sa.get_f(), ra.get_f()) <= 1e-12
    assert rel_l2(sb.get_f(), rb.get_f()) <= 1e-12
    np.testing.assert_allclose(sa.rec[3:5], ra.rec[3:5], rtol=1e-9, atol=1e-12)
    assert len(B.records(ida)) == 3
    ra.close()
    rb.close()
    B.close()
