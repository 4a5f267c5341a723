"""ctypes binding of the C ABI declared in ``include/ilbm_b200.h``.

This is the same binding a host of the library would write; the package's
drivers go through it.  The shared object is
the in-tree ``ilbmrex_b200/lib/libilbm_b200.so``; there is no fallback: if it
cannot be loaded every entry point raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libilbm_b200.so"
MAXQ = 27

ILBM_OK = 0
ILBM_ERR_ARG, ILBM_ERR_CUDA, ILBM_ERR_UNSUPPORTED = -1, -2, -3
ILBM_ERR_NOMEM, ILBM_ERR_SOLVER, ILBM_ERR_RANGE = -4, -5, -6
ILBM_ERR_IO = -7
CKPT_MACRO, CKPT_FORCE, CKPT_BODY = 1, 2, 4
TWO_LEVEL_FIRST_STEP = 1
HIERARCHY_FIRST_STEP = 1
STORAGE = {"f64": 0, "f32": 1, "f16": 2}
GHOST_SELF, GHOST_CALLER = 0, 1
IVC_AUTO, IVC_CG, IVC_DENSE = 0, 1, 2
IVC_DENSE_MAX = 8192
BC_INT_DIR, BC_FOEXTRAP, BC_EXT_DIR, BC_USER_1, BC_USER_2 = 0, 2, 3, 1001, 1002

# every symbol the header declares
EXPORTS = [
    "ilbm_create", "ilbm_destroy", "ilbm_last_error", "ilbm_sync", "ilbm_stream",
    "ilbm_event_record", "ilbm_event_elapsed_ms", "ilbm_kernel_launches", "ilbm_storage_bytes",
    "ilbm_graph_begin", "ilbm_graph_end", "ilbm_graph_launch", "ilbm_graph_destroy",
    "ilbm_level_step", "ilbm_compute_macro", "ilbm_init_equilibrium",
    "ilbm_ib_create", "ilbm_ib_destroy", "ilbm_ib_num_markers", "ilbm_ib_force_region",
    "ilbm_ib_update_forcing", "ilbm_advance_level", "ilbm_ib_last_marker_force_sum",
    "ilbm_ib_solver_stats", "ilbm_ib_set_ivc_solver",
    "ilbm_ib_markers",
    "ilbm_force_integrals", "ilbm_force_integrals_noalloc", "ilbm_force_record_async",
    "ilbm_momentum_exchange",
    "ilbm_batch_create", "ilbm_batch_destroy", "ilbm_batch_add", "ilbm_batch_remove",
    "ilbm_batch_step", "ilbm_batch_case_state", "ilbm_batch_records", "ilbm_batch_set_tiles",
    "ilbm_batch_tune", "ilbm_batch_size", "ilbm_batch_progress",
    "ilbm_derived_fields", "ilbm_tag_cells",
    "ilbm_checkpoint_write", "ilbm_checkpoint_read", "ilbm_plotfile_write",
    "ilbm_advance_two_level", "ilbm_advance_two_level_recorded", "ilbm_average_down",
    "ilbm_advance_hierarchy",
]


class Lattice_t(C.Structure):
    _fields_ = [("dim", C.c_int), ("q", C.c_int),
                ("cx", C.c_double * MAXQ), ("cy", C.c_double * MAXQ), ("cz", C.c_double * MAXQ),
                ("wis", C.c_double * MAXQ), ("wim", C.c_double * MAXQ)]


class Box_t(C.Structure):
    _fields_ = [("lo", C.c_int * 3), ("hi", C.c_int * 3),
                ("ngrow_f", C.c_int), ("ngrow_m", C.c_int),
                ("fstride", C.c_int64 * 3), ("mstride", C.c_int64 * 3),
                ("f_in", C.c_void_p), ("f_out", C.c_void_p),
                ("macro_in", C.c_void_p), ("macro_out", C.c_void_p),
                ("force", C.c_void_p), ("force_prev", C.c_void_p)]


class LevelParams_t(C.Structure):
    _fields_ = [("tau", C.c_double),
                ("domain_lo", C.c_int * 3), ("domain_hi", C.c_int * 3),
                ("periodic", C.c_int * 3),
                ("bc_lo", C.c_int * 3), ("bc_hi", C.c_int * 3),
                ("bc_val_lo", (C.c_double * 4) * 3), ("bc_val_hi", (C.c_double * 4) * 3),
                ("ghost_mode", C.c_int),
                ("use_uniform_force", C.c_int), ("uniform_force", C.c_double * 3),
                ("force_lo", C.c_int * 3), ("force_hi", C.c_int * 3),
                ("f16_scale", C.c_double),
                ("level_boxes", C.POINTER(C.c_int)), ("nlevel_boxes", C.c_int)]


class LevelGeom_t(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_cell", C.c_int * 3),
                ("prob_lo", C.c_double * 3), ("prob_hi", C.c_double * 3),
                ("periodic", C.c_int * 3), ("bc_lo", C.c_int * 3), ("bc_hi", C.c_int * 3),
                ("bc_val_lo", (C.c_double * 4) * 3), ("bc_val_hi", (C.c_double * 4) * 3)]


class IBParams_t(C.Structure):
    _fields_ = [("coupling_method", C.c_int), ("delta_type", C.c_int), ("loop_ns", C.c_int),
                ("mdf_relax", C.c_double), ("explicit_diag_eps", C.c_double),
                ("geometry_type", C.c_int),
                ("box_xlo", C.c_double), ("box_xhi", C.c_double), ("box_ylo", C.c_double),
                ("box_yhi", C.c_double), ("box_zlo", C.c_double), ("box_zhi", C.c_double),
                ("box_ds", C.c_double), ("box_lid_only", C.c_int),
                ("box_lid_ux", C.c_double), ("box_lid_uy", C.c_double), ("box_lid_uz", C.c_double),
                ("box_wall_tol", C.c_double), ("n_marker", C.c_int), ("rd", C.c_double),
                ("ubx", C.c_double), ("uby", C.c_double), ("ubz", C.c_double),
                ("omx", C.c_double), ("omy", C.c_double), ("omz", C.c_double),
                ("ivc_diag_reg", C.c_double), ("ivc_rebuild_matrix", C.c_int),
                ("renormalize_delta", C.c_int),
                ("x0", C.c_double), ("y0", C.c_double), ("z0", C.c_double), ("R", C.c_double),
                ("airfoil_chord", C.c_double), ("airfoil_thickness", C.c_double),
                ("pitch_mean", C.c_double), ("pitch_amplitude", C.c_double),
                ("pitch_frequency", C.c_double), ("pitch_phase", C.c_double),
                ("pivot_x", C.c_double)]


class CheckpointMeta_t(C.Structure):
    _fields_ = [("istep", C.c_int64), ("time", C.c_double), ("user", C.c_double * 16),
                ("flags", C.c_int)]


class PlotInfo_t(C.Structure):
    _fields_ = [("prob_lo", C.c_double * 3), ("prob_hi", C.c_double * 3), ("dx", C.c_double * 3),
                ("time", C.c_double), ("istep", C.c_int), ("levelset", C.c_int),
                ("ls_center", C.c_double * 3), ("ls_radius", C.c_double),
                ("body_u", C.c_double * 3)]


class IlbmError(RuntimeError):
    pass


_lib = None


def lib():
    """Load the library (raises ``IlbmError`` if it is missing or incomplete)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise IlbmError(f"CUDA library not built: {LIB_PATH} (run python -m ilbmrex_b200.build_lib)")
    L = C.CDLL(str(LIB_PATH))
    P, I, D, I64 = C.c_void_p, C.c_int, C.c_double, C.c_int64
    ip3 = C.POINTER(C.c_int)
    dp = C.POINTER(C.c_double)
    sigs = {
        "ilbm_create": (I, [C.POINTER(Lattice_t), I, I, P, C.POINTER(P)]),
        "ilbm_destroy": (I, [P]),
        "ilbm_last_error": (C.c_char_p, []),
        "ilbm_sync": (I, [P]),
        "ilbm_stream": (P, [P]),
        "ilbm_event_record": (I, [P, I]),
        "ilbm_event_elapsed_ms": (I, [P, I, I, C.POINTER(C.c_float)]),
        "ilbm_kernel_launches": (I64, [P]),
        "ilbm_graph_begin": (I, [P]),
        "ilbm_graph_end": (I, [P, C.POINTER(P)]),
        "ilbm_graph_launch": (I, [P, P]),
        "ilbm_graph_destroy": (I, [P]),
        "ilbm_storage_bytes": (I, [P, ip3, ip3]),
        "ilbm_level_step": (I, [P, C.POINTER(Box_t), I, C.POINTER(LevelParams_t)]),
        "ilbm_compute_macro": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t), P, P, P, ip3, ip3]),
        "ilbm_init_equilibrium": (I, [P, C.POINTER(Box_t)]),
        "ilbm_ib_create": (I, [P, C.POINTER(IBParams_t), C.POINTER(LevelGeom_t), C.POINTER(P)]),
        "ilbm_ib_destroy": (I, [P]),
        "ilbm_ib_num_markers": (I, [P, C.POINTER(I64)]),
        "ilbm_ib_force_region": (I, [P, ip3, ip3]),
        "ilbm_ib_update_forcing": (I, [P, C.POINTER(Box_t), I, C.POINTER(LevelParams_t), D, D]),
        "ilbm_advance_level": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t), P, D, D]),
        "ilbm_ib_last_marker_force_sum": (I, [P, dp]),
        "ilbm_ib_solver_stats": (I, [P, C.POINTER(I)]),
        "ilbm_ib_set_ivc_solver": (I, [P, I]),
        "ilbm_ib_markers": (I, [P, dp, dp, dp]),
        "ilbm_force_integrals": (I, [P, C.POINTER(Box_t), I, ip3, ip3, dp]),
        "ilbm_force_integrals_noalloc": (I, [P, C.POINTER(Box_t), P, ip3, ip3, dp]),
        "ilbm_force_record_async": (I, [P, C.POINTER(Box_t), I, P, ip3, ip3, P]),
        "ilbm_batch_create": (I, [P, I, C.POINTER(P)]),
        "ilbm_batch_destroy": (I, [P]),
        "ilbm_batch_add": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t), P, D, D, I,
                               C.POINTER(I)]),
        "ilbm_batch_remove": (I, [P, I]),
        "ilbm_batch_step": (I, [P, I]),
        "ilbm_batch_case_state": (I, [P, I, C.POINTER(I), C.POINTER(I64), dp]),
        "ilbm_batch_records": (I, [P, I, dp, I, C.POINTER(I)]),
        "ilbm_batch_set_tiles": (I, [P, I, I]),
        "ilbm_batch_tune": (I, [P, I, C.POINTER(I), C.POINTER(I), C.POINTER(C.c_float)]),
        "ilbm_batch_size": (I, [P, C.POINTER(I), C.POINTER(I64)]),
        "ilbm_derived_fields": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t), P, P, dp, P, P, dp]),
        "ilbm_tag_cells": (I, [P, C.POINTER(Box_t), P, D, I, dp, dp, D, D, dp, dp, dp, dp, P,
                               C.POINTER(I64)]),
        "ilbm_batch_progress": (I, [P, I, C.POINTER(I), C.POINTER(I64), C.POINTER(I), C.POINTER(I)]),
        "ilbm_advance_two_level": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t), C.POINTER(Box_t),
                                       C.POINTER(LevelParams_t), P, D, D, I]),
        "ilbm_advance_two_level_recorded": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t),
                                                C.POINTER(Box_t), C.POINTER(LevelParams_t), P, D, D,
                                                I, ip3, ip3, P]),
        "ilbm_average_down": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t), C.POINTER(Box_t),
                                  C.POINTER(LevelParams_t)]),
        "ilbm_advance_hierarchy": (I, [P, I, C.POINTER(Box_t), C.POINTER(LevelParams_t), P, D, D, I]),
        "ilbm_checkpoint_write": (I, [P, C.POINTER(Box_t), P, C.POINTER(CheckpointMeta_t), C.c_char_p]),
        "ilbm_checkpoint_read": (I, [P, C.POINTER(Box_t), P, C.POINTER(CheckpointMeta_t), C.c_char_p]),
        "ilbm_plotfile_write": (I, [P, C.POINTER(Box_t), C.POINTER(LevelParams_t),
                                    C.POINTER(PlotInfo_t), C.c_char_p]),
        "ilbm_momentum_exchange": (I, [P, C.POINTER(Box_t), I, C.POINTER(LevelParams_t),
                                       D, D, D, D, dp, dp, I, dp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name)
        fn.restype, fn.argtypes = res, args
    _lib = L
    return L


def check(rc: int, what: str = "") -> None:
    if rc != ILBM_OK:
        msg = lib().ilbm_last_error().decode(errors="replace")
        raise IlbmError(f"{what}: status {rc}: {msg}")


def ivec3(v) -> "C.Array":
    a = (C.c_int * 3)()
    for d in range(3):
        a[d] = int(v[d])
    return a


def dvec3(v) -> "C.Array":
    a = (C.c_double * 3)()
    for d in range(3):
        a[d] = float(v[d])
    return a
