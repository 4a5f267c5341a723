"""The CPU oracle (oracle/lbm_oracle.c) against the reference's own code.

* ``oracle/_ref`` compiles Source/LBM, Source/BC, Source/IBM of the reference
  in place; where it is built the oracle must agree with it bit for bit;
* the committed fixtures in tests/golden were written by that build
  (tests/golden/make_golden.py) and pin the oracle where the reference tree
  is not mounted.
"""
import numpy as np
import pytest

from oracle import checker
from oracle.checker import CpuLevel
from tests.golden.golden_cases import GOLDEN_CASES

GOLDEN = __import__("pathlib").Path(__file__).resolve().parent / "golden"


def _run(backend, name):
    builder, steps = GOLDEN_CASES[name]
    case, init, ib = builder()
    L = CpuLevel(case, backend)
    L.set_macro(*init())
    L.init_equilibrium()
    if ib is not None:
        L.ib_create(ib)
    L.step(steps)
    return L


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_golden_fixture(name):
    """bit-exact: the fixtures are the reference's own outputs"""
    L = _run("oracle", name)
    g = np.load(GOLDEN / f"{name}.npz")
    f = L.get_f()
    np.testing.assert_array_equal(L.get_macro(), g["macro"])
    np.testing.assert_array_equal(L.get_force(), g["force"])
    np.testing.assert_allclose(f.reshape(f.shape[0], -1).sum(axis=1), g["f_sum"], rtol=1e-13, atol=1e-13)
    if "f" in g:
        np.testing.assert_array_equal(f, g["f"])
    if "rec" in g:
        np.testing.assert_array_equal(L.force_record(), g["rec"])
        np.testing.assert_array_equal(L.marker_force_sum(), g["fsum"])
        assert L.num_markers() == int(g["nmark"])


@pytest.mark.parametrize("name", sorted(GOLDEN_CASES))
def test_oracle_matches_reference_build(name):
    case = GOLDEN_CASES[name][0]()[0]
    if not checker.available("ref", case.dim):
        pytest.skip("reference build (oracle/_ref/libref*.so) not present")
    a, b = _run("oracle", name), _run("ref", name)
    np.testing.assert_array_equal(a.get_f(), b.get_f())
    np.testing.assert_array_equal(a.get_macro(), b.get_macro())


def test_delta_kernel_matches_reference_and_partitions_unity():
    """IBMarkerDF.cpp:70-99; the 4-point and 3-point kernels sum to 1/h and
    have first moment 0 on a uniform grid (the reference's own
    debug_kernel_partition diagnostic, IBMarkerDF.cpp:1585-1689)."""
    lib = checker._load("oracle", 2)
    rng = np.random.default_rng(20261203)
    for kt in (0, 1):
        for _ in range(50):
            xp = rng.uniform(0, 1)
            h = 1.0
            xs = np.arange(-3, 5) + 0.5
            vals = np.array([lib.orc_delta_function(x, xp, h, kt) for x in xs])
            assert abs(vals.sum() * h - 1.0) < 1e-14
            assert abs(np.sum(vals * (xs - xp)) * h) < 1e-14
    if checker.available("ref", 2):
        ref = checker._load("ref", 2)
        for x in np.linspace(-2.5, 2.5, 101):
            for kt in (0, 1):
                assert ref.ref_delta_function(x, 0.1, 1.0, kt) == lib.orc_delta_function(x, 0.1, 1.0, kt)


@pytest.mark.parametrize("name", ["cylinder96x64_ivc", "sphere40x24x24_d3q19_ivc",
                                  "channel16x12_bounceback", "duct12_d3q19_user2",
                                  "couette24_extdir_foextrap"])
def test_derived_and_tags_match_reference_build(name):
    """The numpy restatements of visPara and ErrorEst's tagging (which check
    the device kernels) against the reference's own visPara.H, Tagging.H and
    LevelSet.cpp compiled in place, on the oracle's FillPatched macro."""
    from ilbmrex_b200.level import refinement_region
    case, init, ib = GOLDEN_CASES[name][0]()
    if not checker.available("ref", case.dim):
        pytest.skip("reference build (oracle/_ref/libref*.so) not present")
    a, b = _run("oracle", name), _run("ref", name)
    ng = case.nghost
    nx, ny, nz = case.n_cell
    gz = nz + 2 * ng if case.dim == 3 else 1
    mg = a.fill_patch_macro().reshape(6, gz, ny + 2 * ng, nx + 2 * ng)
    vor, pres = checker.vorticity_pressure(mg, ng, case.dim, case.dx, case.dx, case.dx)
    rv, rp, rmax = b.ref_derived()
    np.testing.assert_array_equal(vor, rv)
    np.testing.assert_array_equal(pres, rp)
    assert vor.max() == rmax
    box = refinement_region(case, ib) if ib is not None else None
    ls = (ib.x0, ib.y0, ib.z0 if case.dim == 3 else 0.0, ib.R, 5, case.dx) if ib is not None else None
    for ratio, nr, bx, l6 in ((0.3, (0.0, 0.0), box, ls), (0.05, (4.0, 6.0), box, ls),
                              (0.3, (0.0, 0.0), None, ls), (0.1, (0.0, 0.0), box, None)):
        mine = checker.error_est_tags(vor, ratio * rmax, case.prob_lo, case.prob_hi, [case.dx] * 3,
                                      bx, nr, l6)
        ref = b.ref_tags(rv, ratio * rmax, bx, nr, l6)
        np.testing.assert_array_equal(mine, ref)
        assert ref.sum() > 0 or nr != (0.0, 0.0)


def test_two_level_oracle_invariants():
    """The oracle's two-level driver: a uniform state stays uniform across the
    coarse-fine boundary, and after a step every covered coarse cell holds the
    mean of its four fine cells (average-down)."""
    from ilbmrex_b200 import cases
    from oracle.checker import CpuTwoLevel
    c = cases.LevelCase(cases.D2Q9, (24, 24, 1), nu=0.02)
    tl = cases.TwoLevelCase(c, (12, 12), (35, 35))
    T = CpuTwoLevel(tl)
    T.set_macro(0, *cases.uniform_init(c, 1.0, (0.03, -0.01, 0.0))())
    T.set_macro(1, *cases.uniform_init(tl.fine_box(), 1.0, (0.03, -0.01, 0.0))())
    T.init_equilibrium()
    T.step(4)
    for lev in (0, 1):
        m = T.get_macro(lev)
        assert np.abs(m[1] - 0.03).max() < 1e-14 and np.abs(m[2] + 0.01).max() < 1e-14
    tl2, ic, if_ = cases.shear_layer_two_level(n=32, fine=(16, 48))
    T2 = CpuTwoLevel(tl2)
    T2.set_macro(0, *ic())
    T2.set_macro(1, *if_())
    T2.init_equilibrium()
    T2.step(3)
    fc, ff = T2.get_f(0), T2.get_f(1)
    sub = ff[:, 0]
    mean = 0.25 * (((sub[:, 0::2, 0::2] + sub[:, 0::2, 1::2]) + sub[:, 1::2, 0::2]) + sub[:, 1::2, 1::2])
    np.testing.assert_array_equal(fc[:, 0, 8:24, 8:24], mean)


def test_spreading_order_sensitivity():
    """How much the reference's own result depends on the marker order of its
    force spreading (the device spreads with FP64 atomics in an unspecified
    order): below 1e-15 relative for explicit and IVC coupling, above 1e-12
    for explicit_diag, whose division by the operator's small diagonal
    amplifies rounding (the GPU parity test allows that measured change)."""
    def run(name, rev):
        checker.set_spread_order(rev)
        try:
            return _run("oracle", name).get_f()
        finally:
            checker.set_spread_order(False)
    for name in ("cylinder96x64_ivc", "cylinder96x64_explicit_mdf2", "sphere40x24x24_d3q19_ivc"):
        a, b = run(name, False), run(name, True)
        assert np.sqrt(np.sum((a - b) ** 2) / np.sum(a ** 2)) < 1e-15, name
    a, b = run("cylinder96x64_explicit_diag_mdf2", False), run("cylinder96x64_explicit_diag_mdf2", True)
    assert np.sqrt(np.sum((a - b) ** 2) / np.sum(a ** 2)) > 1e-12
