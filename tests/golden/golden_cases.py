"""Small cases whose reference outputs are stored as golden fixtures."""
from __future__ import annotations

from ilbmrex_b200 import cases


def _tgv():
    c, init = cases.taylor_green(32, U0=0.01, tau=0.8)
    return c, init, None


def _couette():
    c, init = cases.couette(24, U=0.1, nu=0.064)
    return c, init, None


def _channel():
    c, init = cases.channel_bounce_back(16, 12, force=1.0e-5, nu=0.1)
    return c, init, None


def _duct():
    c, init = cases.square_duct(N=12, L=4, force=1.0e-5, nu=0.06)
    return c, init, None


def _cylinder_ivc():
    c, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    return c, init, ib


def _cylinder_explicit():
    c, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40,
                                 coupling=0)
    ib.loop_ns = 2
    return c, init, ib


def _sphere_ivc():
    c, ib, init = cases.sphere(nx=40, ny=24, nz=24, D=8, center=(12.2, 11.7, 12.4), U=0.04, Re=20)
    return c, init, ib


def _cavity_lid():
    c, ib, init = cases.cavity_lid(32)
    return c, init, ib


def _airfoil():
    # the reference's own pitching-airfoil constants (leading-edge pivot)
    from ilbmrex_b200.cases import D2Q9, EXT_DIR, FOEXTRAP, INT_DIR, LevelCase, MarkerIB
    case = LevelCase(D2Q9, (96, 64, 1), periodic=(False, True, True),
                     bc_lo=(EXT_DIR, INT_DIR, INT_DIR), bc_hi=(FOEXTRAP, INT_DIR, INT_DIR),
                     bc_lo_val=((1.0, 0.05, 0.0, 0.0), (0.0,) * 4, (0.0,) * 4), nu=0.02,
                     name="airfoil_ref")
    ib = MarkerIB(coupling_method=1, delta_type=4, geometry_type=2, ivc_diag_reg=1.3,
                  x0=30.0, y0=32.0, R=10.0, U0=0.05, airfoil=MarkerIB.AIRFOIL_DEFAULT)
    return case, cases.uniform_init(case, 1.0, (0.05, 0.0, 0.0)), ib


def _cylinder_delta3():
    # 3-point kernel (IBMarkerDF.cpp:86-96) with IVC coupling
    c, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    ib.delta_type = 3
    return c, init, ib


def _cylinder_explicit_diag():
    # explicit_diag coupling (IBMarkerDF.cpp:745-865): (U_d - U) / (dt * M_kk)
    c, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40,
                                 coupling=2)
    ib.loop_ns = 2
    return c, init, ib


def _cylinder_ivc_renorm():
    # renormalize_delta with IVC: spreading renormalised, interpolation not
    # (IBMarkerDF.cpp:541-542, 727-728, 1484).  No stencil is clipped in these
    # renorm cases, so each weight is divided by a partition of one up to
    # rounding: the fixtures pin that arithmetic bit for bit.
    c, ib, init = cases.cylinder(nx=96, ny=64, D=16, center=(32.3, 31.7), U=0.05, Re=40)
    ib.renormalize_delta = 1
    return c, init, ib


def _cavity_lid_renorm():
    # renormalize_delta with explicit coupling: interpolation and spreading
    # renormalised, 3-point kernel, lid markers along the cavity's top
    c, ib, init = cases.cavity_lid(32)
    ib.renormalize_delta = 1
    ib.delta_type = 3
    return c, init, ib


def _sphere_delta3_diag():
    # 3D: 3-point kernel with explicit_diag coupling, two MDF iterations
    c, ib, init = cases.sphere(nx=40, ny=24, nz=24, D=8, center=(12.2, 11.7, 12.4), U=0.04, Re=20,
                               coupling=2)
    ib.delta_type = 3
    ib.loop_ns = 2
    return c, init, ib


GOLDEN_CASES = {
    "tgv32_d2q9": (_tgv, 20),
    "couette24_extdir_foextrap": (_couette, 20),
    "channel16x12_bounceback": (_channel, 20),
    "duct12_d3q19_user2": (_duct, 10),
    "cylinder96x64_ivc": (_cylinder_ivc, 8),
    "cylinder96x64_explicit_mdf2": (_cylinder_explicit, 8),
    "sphere40x24x24_d3q19_ivc": (_sphere_ivc, 4),
    "cavity32_lid_box": (_cavity_lid, 8),
    "airfoil96x64_pitching_ivc": (_airfoil, 6),
    "cylinder96x64_delta3_ivc": (_cylinder_delta3, 8),
    "cylinder96x64_explicit_diag_mdf2": (_cylinder_explicit_diag, 8),
    "cylinder96x64_ivc_renorm": (_cylinder_ivc_renorm, 8),
    "cavity32_lid_renorm_delta3": (_cavity_lid_renorm, 8),
    "sphere40x24x24_delta3_diag": (_sphere_delta3_diag, 4),
}
