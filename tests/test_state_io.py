"""State I/O through the C ABI: checkpoint / restart and the AMReX plotfile.

* A checkpoint restores the saved state bit for bit (populations, F^{n-1},
  the stored macro fields of a level that has not stepped yet, the body's
  markers and CG start vector), and the restarted run continues the saved one:
  bit for bit without a body; with a body the marker forces are spread with
  FP64 atomics in no fixed order, so two runs of the same state agree to
  1e-12 (FP64) / 1e-5 (FP32) relative L2, the bound every IB parity test uses.
* A file that does not match the context, box or body, a truncated file and a
  flipped byte are refused with ILBM_ERR_ARG / ILBM_ERR_IO.
* The plotfile read back with ilbmrex_b200.plotfile equals the level's own
  read-backs: macro fields, vorticity and pressure, unshifted populations, the
  body's level set and PlotFileMF's masking of the body interior.
"""
import numpy as np
import pytest

from ilbmrex_b200 import capi, cases
from ilbmrex_b200.plotfile import plotfile_name, read_plotfile

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("needs a CUDA device", allow_module_level=True)

from ilbmrex_b200.batch import Batch  # noqa: E402
from ilbmrex_b200.lattice import D2Q9  # noqa: E402
from ilbmrex_b200.level import LevelSolver  # noqa: E402


def rel_l2(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / max(np.sum(b ** 2), 1e-300)))


def _case(which):
    if which == "cylinder":
        c, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    elif which == "airfoil":
        c, ib, init = cases.pitching_airfoil(nx=128, ny=96, chord=32.0, pivot=(40.0, 48.0), U=0.05,
                                             Re=80.0, amplitude_deg=8.0, reduced_frequency=0.2)
    elif which == "sphere":
        c, ib, init = cases.sphere(48, 32, 32, D=12.0, center=(16.3, 15.8, 16.1), U=0.04, Re=40.0)
    elif which == "channel":
        (c, init), ib = cases.channel_bounce_back(nx=40, ny=24), None
    else:
        (c, init), ib = cases.square_duct(N=10, L=6, force=1e-4, nu=0.06), None
    return c, ib, init


def _solver(which, storage):
    c, ib, init = _case(which)
    s = LevelSolver(c, storage, ib=ib)
    s.set_macro(*init())
    return s


@pytest.mark.parametrize("which,storage", [("channel", "f64"), ("duct", "f32"), ("channel", "f16"),
                                           ("cylinder", "f64"), ("airfoil", "f64"),
                                           ("sphere", "f32")])
def test_checkpoint_restart(which, storage, tmp_path):
    n0, n1 = 6, 5
    a = _solver(which, storage)
    a.step(n0, record_force=a.ib is not None)
    path = tmp_path / "chk00006"
    a.save_checkpoint(path)
    f_saved = a.get_f()
    F_saved = a.get_force() if a.ib is not None else None
    mk_saved = a.markers() if a.ib is not None else None

    b = LevelSolver(*_case(which)[:1], storage, ib=_case(which)[1])
    b.load_checkpoint(path)
    assert b.istep == a.istep == n0 and b.time == a.time
    assert b.have_prev_body == a.have_prev_body
    np.testing.assert_array_equal(b.prev_body, a.prev_body)
    np.testing.assert_array_equal(b.get_f(), f_saved)
    if a.ib is not None:
        np.testing.assert_array_equal(b.get_force(), F_saved)
        for x, y in zip(b.markers(), mk_saved):
            np.testing.assert_array_equal(x, y)
        np.testing.assert_array_equal(b.marker_force_sum(), a.marker_force_sum())

    a.step(n1, record_force=a.ib is not None)
    b.step(n1, record_force=b.ib is not None)
    if a.ib is None:
        np.testing.assert_array_equal(b.get_f(), a.get_f())
    else:
        tol = 1e-12 if storage == "f64" else 1e-5
        assert rel_l2(b.get_f(), a.get_f()) <= tol
        np.testing.assert_allclose(b.rec[3:5], a.rec[3:5], rtol=1e-9 if storage == "f64" else 1e-4,
                                   atol=1e-12)
    a.close()
    b.close()


def test_checkpoint_restart_grid_cg(tmp_path):
    """A body solved every step by the grid-wide CG (more than 1024 markers)
    restarts with its CG start vectors (the last solution and the one before
    it, for the extrapolated start) and continues the saved run."""
    c, ib, init = cases.sphere(64, 48, 48, D=24.0, center=(24.3, 23.8, 24.1), U=0.04, Re=40.0)
    a = LevelSolver(c, "f64", ib=ib)
    a.set_ivc_solver(capi.IVC_CG)
    a.set_macro(*init())
    assert a.num_markers() > 1024
    a.step(6, record_force=True)
    path = tmp_path / "chk_cg"
    a.save_checkpoint(path)
    b = LevelSolver(c, "f64", ib=cases.sphere(64, 48, 48, D=24.0, center=(24.3, 23.8, 24.1), U=0.04,
                                              Re=40.0)[1])
    b.set_ivc_solver(capi.IVC_CG)
    b.load_checkpoint(path)
    assert b.istep == 6
    a.step(5, record_force=True)
    b.step(5, record_force=True)
    assert a.cg_iterations() > 0 and b.cg_iterations() > 0
    assert rel_l2(b.get_f(), a.get_f()) <= 1e-12
    np.testing.assert_allclose(b.rec[3:5], a.rec[3:5], rtol=1e-9, atol=1e-12)
    a.close()
    b.close()


def test_checkpoint_before_the_first_step(tmp_path):
    """A level saved right after initialisation carries its stored macro
    fields (the first step reads them): the restart takes the same first step."""
    a = _solver("channel", "f64")
    path = tmp_path / "chk00000"
    a.save_checkpoint(path)
    b = LevelSolver(_case("channel")[0], "f64")
    b.load_checkpoint(path)
    assert b.first_step_macro and b.istep == 0
    a.step(3)
    b.step(3)
    np.testing.assert_array_equal(b.get_f(), a.get_f())
    a.close()
    b.close()


def test_restored_case_joins_a_batch(tmp_path):
    """A case checkpointed out of a batch and restored into a fresh solver
    rejoins another batch and continues like the uninterrupted run."""
    c, ib, init = _case("cylinder")
    B = Batch(D2Q9, "f64")
    cid = B.add(B.solver(c, ib, init), max_steps=64)
    B.step(5)
    s = B.sync(cid)
    path = tmp_path / "case.chk"
    s.save_checkpoint(path)
    B.step(6)
    ref = B.sync(cid)
    B2 = Batch(D2Q9, "f64")
    r = B2.solver(c, ib, None)
    r.load_checkpoint(path)
    assert r.istep == 6
    cid2 = B2.add(r, max_steps=64)  # takes its first step since the restart alone
    assert r.istep == 7
    B2.step(5)
    r = B2.sync(cid2)
    assert r.istep == ref.istep == 12
    assert rel_l2(r.get_f(), ref.get_f()) <= 1e-12
    B.close()
    B2.close()


def test_checkpoint_refusals(tmp_path):
    a = _solver("cylinder", "f64")
    a.step(2)
    path = tmp_path / "chk"
    a.save_checkpoint(path)
    raw = path.read_bytes()
    # another storage form, another box, no body
    for other in (LevelSolver(_case("cylinder")[0], "f32", ib=_case("cylinder")[1]),
                  LevelSolver(cases.cylinder(nx=80, ny=64, D=16, center=(32.3, 31.7), U=0.05,
                                             Re=40)[0], "f64", ib=_case("cylinder")[1]),
                  LevelSolver(_case("cylinder")[0], "f64")):
        with pytest.raises(capi.IlbmError) as e:
            other.load_checkpoint(path)
        assert "ilbm_checkpoint_read" in str(e.value)
        other.close()
    b = LevelSolver(_case("cylinder")[0], "f64", ib=_case("cylinder")[1])
    bad = bytearray(raw)
    bad[len(bad) // 2] ^= 0x40
    (tmp_path / "flip").write_bytes(bytes(bad))
    with pytest.raises(capi.IlbmError) as e:
        b.load_checkpoint(tmp_path / "flip")
    assert "hash mismatch" in str(e.value)
    (tmp_path / "short").write_bytes(raw[: len(raw) - 1000])
    with pytest.raises(capi.IlbmError) as e:
        b.load_checkpoint(tmp_path / "short")
    assert "short file" in str(e.value)
    with pytest.raises(capi.IlbmError):
        b.load_checkpoint(tmp_path / "missing")
    b.load_checkpoint(path)  # the good file still loads into the same solver
    np.testing.assert_array_equal(b.get_f(), a.get_f())
    a.close()
    b.close()


@pytest.mark.parametrize("which,storage", [("cylinder", "f64"), ("sphere", "f32"),
                                           ("channel", "f16"), ("duct", "f64")])
def test_plotfile(which, storage, tmp_path):
    s = _solver(which, storage)
    s.step(4)
    d = tmp_path / plotfile_name("plt", s.istep)
    s.write_plotfile(d)
    pf = read_plotfile(d)
    c = s.case
    q = c.lattice.q
    ls = s.ib_case is not None and s.ib_case.geometry_type == 0
    assert pf.names[:6] == ["rho", "ux", "uy", "uz", "vor", "Pressure"]
    assert pf.names[6:6 + q] == [f"f_new_{i}" for i in range(q)]
    assert pf.names[6 + q:] == (["phi"] if ls else [])
    assert pf.dim == c.dim and pf.time == s.time and pf.level_steps == [s.istep]
    assert pf.dx == tuple([c.dx] * c.dim)
    assert pf.domain[1] == tuple(n - 1 for n in c.n_cell[:c.dim])
    f = s.get_f()
    for i in range(q):
        np.testing.assert_array_equal(pf.data[f"f_new_{i}"], f[i])
    mac = s.get_macro()
    vor, pres, _ = s.derived_fields()
    inside = np.zeros(c.shape, dtype=bool)
    if ls:
        m = s.ib_case
        nz, ny, nx = c.shape
        k, j, i = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
        x = c.prob_lo[0] + (i + 0.5) * c.dx
        y = c.prob_lo[1] + (j + 0.5) * c.dx
        r2 = (x - m.x0) * (x - m.x0) + (y - m.y0) * (y - m.y0)
        if c.dim == 3:
            z = c.prob_lo[2] + (k + 0.5) * c.dx
            r2 = r2 + (z - m.z0) * (z - m.z0)
        phi = np.sqrt(r2) - m.R
        np.testing.assert_array_equal(pf.data["phi"], phi)
        inside = phi < 0.0
        assert inside.any()
    np.testing.assert_array_equal(pf.data["rho"], mac[0])
    np.testing.assert_array_equal(pf.data["Pressure"], pres)
    ub = (s.ib_case.ubx, s.ib_case.uby, s.ib_case.ubz) if ls else (0.0, 0.0, 0.0)
    for n, name in enumerate(("ux", "uy", "uz")):
        want = mac[1 + n] if (n < 2 or c.dim == 3) else np.zeros(c.shape)
        np.testing.assert_array_equal(pf.data[name], np.where(inside, ub[n], want))
    np.testing.assert_array_equal(pf.data["vor"], np.where(inside, 0.0, vor))
    for n, name in enumerate(pf.names):
        assert pf.cell_min[n] == pf.data[name].min() and pf.cell_max[n] == pf.data[name].max()
    s.close()
