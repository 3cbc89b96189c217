"""ctypes bindings of include/tpicb200.h (the library's C ABI).

The library is the in-tree tpic_b200/libtpicb200.so built for sm_100a by
tpic_b200/build.py. Loading fails loudly when it is missing: there is no
Python or CPU fallback for any stage of the cycle.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIBRARY = Path(__file__).resolve().parent / "libtpicb200.so"

SUCCESS, INVALID_ARGUMENT, INVALID_STATE, OVERFLOW, BACKEND_FAILURE = 0, 1, 2, 3, 4
NOT_CONVERGED, CAPACITY_EXCEEDED, INVALID_DATA = 5, 6, 7
PRECISION_DOUBLE, PRECISION_MIXED = 0, 1
MASS_SCALAR, MASS_SCALAR_F64, MASS_TF32, MASS_BF16X3, MASS_MOMENTS_F64 = 0, 1, 2, 3, 4
MASS_LAYOUT_RECORDS, MASS_LAYOUT_STENCIL_MAJOR, MASS_LAYOUT_TILED = 0, 1, 2
STALL_NONE, STALL_DEPOSIT, STALL_APPLY = 0, 1, 2
MAX_SPECIES = 8

MASS_KINDS = {"scalar": MASS_SCALAR, "scalar-f64": MASS_SCALAR_F64, "fp64": MASS_SCALAR_F64,
              "tf32": MASS_TF32, "bf16x3": MASS_BF16X3, "matrix-core": MASS_TF32,
              "moments-f64": MASS_MOMENTS_F64}
PRECISIONS = {"double": PRECISION_DOUBLE, "mixed": PRECISION_MIXED}


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double)]


class Options(C.Structure):
    _fields_ = [("dt", C.c_double), ("theta", C.c_double), ("c", C.c_double), ("gmres_tol", C.c_double),
                ("gmres_restart", C.c_int), ("gmres_max_iterations", C.c_int), ("precision", C.c_int),
                ("max_particles", C.c_uint32), ("mass_layout", C.c_int), ("smooth_iterations", C.c_int),
                ("smooth_alpha", C.c_double), ("smooth_operator", C.c_int)]


class Particles(C.Structure):
    _fields_ = [("rx", C.c_void_p), ("ry", C.c_void_p), ("rz", C.c_void_p),
                ("u", C.c_void_p), ("v", C.c_void_p), ("w", C.c_void_p),
                ("q", C.c_void_p), ("cell", C.c_void_p), ("id", C.c_void_p), ("count", C.c_uint32)]


class Layout(C.Structure):
    _fields_ = [("node_count", C.c_int64), ("cell_count", C.c_int64), ("bin_count", C.c_int64),
                ("interior_nodes", C.c_int64), ("field_scalar_bytes", C.c_size_t),
                ("mass_scalar_bytes", C.c_size_t), ("velocity_scalar_bytes", C.c_size_t),
                ("mass_count", C.c_int64)]


class GmresResult(C.Structure):
    _fields_ = [("converged", C.c_int), ("iterations", C.c_int), ("initial_residual", C.c_double),
                ("residual", C.c_double), ("rhs_norm", C.c_double), ("relative_residual", C.c_double),
                ("host_waits", C.c_int)]


class State(C.Structure):
    _fields_ = [("ns", C.c_int), ("qom", C.c_double * MAX_SPECIES),
                ("slot", (Particles * 2) * MAX_SPECIES), ("current", C.c_int * MAX_SPECIES),
                ("counts", C.c_void_p * MAX_SPECIES), ("offsets", C.c_void_p * MAX_SPECIES),
                ("e", C.c_void_p), ("b_cell", C.c_void_p), ("b_node", C.c_void_p),
                ("b_cell_next", C.c_void_p), ("b_node_next", C.c_void_p), ("j", C.c_void_p),
                ("mass", C.c_void_p), ("e_theta", C.c_void_p), ("mass_kind", C.c_int),
                ("ranks", C.c_void_p * MAX_SPECIES), ("ranked", C.c_int * MAX_SPECIES)]


class CycleReport(C.Structure):
    _fields_ = [("gmres", GmresResult), ("field_energy", C.c_double * 2),
                ("species", (C.c_double * 5) * MAX_SPECIES), ("total_energy", C.c_double),
                ("stage_ms", C.c_float * 6)]


class Adjoint(C.Structure):
    _fields_ = [("ns", C.c_int), ("e_bar", C.c_void_p), ("b_bar", C.c_void_p),
                ("x_bar", C.c_void_p * MAX_SPECIES), ("v_bar", C.c_void_p * MAX_SPECIES),
                ("q_bar", C.c_void_p * MAX_SPECIES), ("count", C.c_uint32 * MAX_SPECIES),
                ("e_theta_bar", C.c_void_p), ("lambda_", C.c_void_p), ("b_node_bar", C.c_void_p),
                ("b_node", C.c_void_p), ("j", C.c_void_p), ("mass", C.c_void_p)]


class Tape(C.Structure):
    _fields_ = [("ns", C.c_int), ("qom", C.c_double * MAX_SPECIES), ("species", Particles * MAX_SPECIES),
                ("counts", C.c_void_p * MAX_SPECIES), ("offsets", C.c_void_p * MAX_SPECIES),
                ("e", C.c_void_p), ("b_cell", C.c_void_p), ("e_theta", C.c_void_p), ("mass_kind", C.c_int)]


CASE_NAME_MAX = 32


class DeckSpecies(C.Structure):
    _fields_ = [("rho", C.c_double), ("qom", C.c_double), ("vth", C.c_double * 3), ("drift", C.c_double * 3),
                ("npcel", C.c_int * 3), ("center_velocity", C.c_int)]


class Deck(C.Structure):
    _fields_ = [("case_name", C.c_char * CASE_NAME_MAX), ("grid", Grid),
                ("dt", C.c_double), ("theta", C.c_double), ("c", C.c_double), ("gmres_tol", C.c_double),
                ("ncycles", C.c_int), ("ns", C.c_int), ("species", DeckSpecies * MAX_SPECIES),
                ("b0", C.c_double * 3), ("delta", C.c_double), ("harris_b0x", C.c_double),
                ("pert_gem", C.c_double), ("pert_hump", C.c_double), ("deltax_hump", C.c_double),
                ("deltay_hump", C.c_double), ("kx_hump", C.c_double), ("ky_hump", C.c_double),
                ("weibel_mode_x", C.c_int), ("weibel_amplitude", C.c_double), ("weibel_growth_rate", C.c_double),
                ("two_stream_mode_x", C.c_int), ("two_stream_amplitude", C.c_double),
                ("two_stream_phase", C.c_double), ("quiet_start", C.c_int), ("ignored_keys", C.c_int),
                ("smooth_iterations", C.c_int), ("smooth_alpha", C.c_double), ("smooth_operator", C.c_int)]


class CheckpointInfo(C.Structure):
    _fields_ = [("version", C.c_int), ("precision", C.c_int), ("cycle", C.c_int), ("ns", C.c_int), ("grid", Grid),
                ("dt", C.c_double), ("c", C.c_double), ("qom", C.c_double * MAX_SPECIES),
                ("count", C.c_uint32 * MAX_SPECIES), ("has_id", C.c_int * MAX_SPECIES)]



class VtkSpecies(C.Structure):
    _fields_ = [("count", C.c_uint64), ("position", C.c_void_p), ("velocity", C.c_void_p), ("charge", C.c_void_p),
                ("id", C.c_void_p), ("species", C.c_uint64)]


EXPORTS = {
    "tpicb200_version": (C.c_char_p, []),
    "tpicb200_last_error": (C.c_char_p, []),
    "tpicb200_launch_count": (C.c_ulonglong, []),
    "tpicb200_create": (C.c_int, [C.POINTER(Grid), C.POINTER(Options), C.POINTER(C.c_void_p)]),
    "tpicb200_destroy": (C.c_int, [C.c_void_p]),
    "tpicb200_get_layout": (C.c_int, [C.c_void_p, C.POINTER(Layout)]),
    "tpicb200_mover": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                 C.c_void_p, C.c_void_p]),
    "tpicb200_sort": (C.c_int, [C.c_void_p, C.POINTER(Particles), C.POINTER(Particles), C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_sort_binned": (C.c_int, [C.c_void_p, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                       C.POINTER(Particles), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_sort_static": (C.c_int, [C.POINTER(Grid), C.c_int, C.POINTER(Particles), C.POINTER(Particles),
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_clear_moments": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_deposit": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "tpicb200_deposit_species": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(Particles),
                                           C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "tpicb200_fold_periodic": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_mass_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_field_solve": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.POINTER(GmresResult), C.c_void_p]),
    "tpicb200_field_advance": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]),
    "tpicb200_magnetic_to_nodes": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_smooth": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_read_invalid": (C.c_int, [C.c_void_p, C.POINTER(C.c_uint32), C.c_int, C.c_void_p]),
    "tpicb200_set_wait_limit": (C.c_int, [C.c_void_p, C.c_uint32]),
    "tpicb200_inject_stall": (C.c_int, [C.c_void_p, C.c_int, C.c_uint32]),
    "tpicb200_energy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(Particles),
                                  C.POINTER(C.c_double), C.c_int, C.POINTER(C.c_double), C.c_void_p]),
    "tpicb200_prepare": (C.c_int, [C.c_void_p, C.POINTER(State), C.c_void_p]),
    "tpicb200_materialize": (C.c_int, [C.c_void_p, C.POINTER(State), C.c_void_p]),
    "tpicb200_deck_parse": (C.c_int, [C.c_char_p, C.POINTER(Deck)]),
    "tpicb200_case_fields": (C.c_int, [C.POINTER(Deck), C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                                       C.c_void_p, C.c_void_p]),
    "tpicb200_case_profile": (C.c_int, [C.POINTER(Deck), C.c_int, C.c_longlong, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_cycle": (C.c_int, [C.c_void_p, C.POINTER(State), C.c_int, C.POINTER(CycleReport), C.c_void_p]),
    "tpicb200_load_species": (C.c_int, [C.c_void_p, C.POINTER(Deck), C.c_int, C.c_uint64, C.c_uint64,
                                        C.POINTER(Particles), C.c_void_p, C.c_void_p]),
    "tpicb200_center_velocities": (C.c_int, [C.c_void_p, C.POINTER(Deck), C.c_int, C.POINTER(Particles), C.c_void_p,
                                             C.c_void_p]),
    "tpicb200_cycle_forward": (C.c_int, [C.c_void_p, C.POINTER(State), C.POINTER(Tape), C.POINTER(CycleReport),
                                         C.c_void_p]),
    "tpicb200_cycle_backward": (C.c_int, [C.c_void_p, C.POINTER(Tape), C.POINTER(Adjoint), C.POINTER(GmresResult),
                                          C.c_void_p]),
    "tpicb200_adjoint_energy": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                          C.POINTER(Adjoint), C.c_void_p]),
    "tpicb200_field_advance_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_mover_backward": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                          C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_void_p]),
    "tpicb200_deposit_backward": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                            C.c_double, C.c_void_p, C.c_void_p, C.c_double, C.c_uint32, C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_field_solve_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.POINTER(GmresResult), C.c_void_p]),
    "tpicb200_magnetic_to_nodes_backward": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tpicb200_checkpoint_write": (C.c_int, [C.c_void_p, C.POINTER(State), C.c_char_p, C.c_int, C.c_void_p]),
    "tpicb200_checkpoint_find": (C.c_int, [C.c_char_p, C.c_char_p, C.c_size_t]),
    "tpicb200_checkpoint_info_read": (C.c_int, [C.c_char_p, C.POINTER(CheckpointInfo)]),
    "tpicb200_checkpoint_read": (C.c_int, [C.c_void_p, C.POINTER(State), C.c_char_p, C.POINTER(CheckpointInfo),
                                           C.c_void_p]),
    "tpicb200_output_moments": (C.c_int, [C.c_void_p, C.c_double, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    "tpicb200_output_particles": (C.c_int, [C.c_void_p, C.POINTER(Particles), C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p]),
    "tpicb200_vtk_write_field": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(Grid), C.c_void_p, C.c_int,
                                           C.c_double, C.c_int, C.c_char_p, C.c_char_p, C.c_int]),
    "tpicb200_vtk_write_particles": (C.c_int, [C.c_char_p, C.c_int, C.c_double, C.c_int, C.c_char_p, C.c_char_p,
                                               C.c_int, C.POINTER(VtkSpecies), C.c_int]),
    "tpicb200_vtk_write_cells": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(Grid), C.c_void_p, C.c_int, C.c_double,
                                           C.c_int, C.c_char_p, C.c_char_p, C.c_int]),
    "tpicb200_gauss_field": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                       C.c_int, C.c_void_p, C.c_void_p]),
    "tpicb200_gauss_charge": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Particles), C.c_void_p, C.c_void_p,
                                        C.c_void_p]),
}

_lib = None


class TpicError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"tpicb200 status {status}: {message}")
        self.status = status


def load() -> C.CDLL:
    """Loads the sm_100a library; raises when it has not been built."""
    global _lib
    if _lib is None:
        if not LIBRARY.exists():
            raise RuntimeError(f"{LIBRARY} is missing: run `python -m tpic_b200.build` (no CPU fallback exists)")
        lib = C.CDLL(str(LIBRARY))
        for name, (restype, argtypes) in EXPORTS.items():
            fn = getattr(lib, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _lib = lib
    return _lib


def check(status: int) -> None:
    if status != SUCCESS:
        message = load().tpicb200_last_error().decode()
        raise TpicError(status, message)
