"""ctypes binding of libpd_b200.so (the C ABI declared in include/pd_b200.h).

The library is built in-tree by ``peridigm_b200.build.build()``. There is no
CPU fallback: if the shared library is missing or cannot be loaded, importing
the compute entry points raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpd_b200.so")

PD_OK = 0
PD_ERR_ARG = 1
PD_ERR_CUDA = 2
PD_ERR_NONFINITE = 3
PD_ERR_TIMEOUT = 4
PD_ERR_STATE = 5
PD_ERR_UNSUPPORTED = 6
PD_ERR_NOMEM = 7
PD_ERR_NOT_CONVERGED = 8

PD_FP64 = 0
PD_SPLIT_FP32 = 1
PD_FP64_SLICED = 2

FIELDS = {
    "Displacement": 0,
    "Velocity": 1,
    "Acceleration": 2,
    "Force_Density": 3,
    "Contact_Force_Density": 4,
    "Dilatation": 5,
    "Weighted_Volume": 6,
    "Damage": 7,
    "Bond_Damage": 8,
    "Coordinates": 9,
    "Number_Of_Neighbors": 10,
    "Force": 11,
    "Volume": 12,
    "Model_Coordinates": 13,
}

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)
_vp = C.c_void_p


class Config(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("influence", C.c_int),
                ("threads_per_point", C.c_int)]


class PlaneFilter(C.Structure):
    _fields_ = [("normal", C.c_double * 3), ("lower_left", C.c_double * 3), ("bottom_unit", C.c_double * 3),
                ("bottom_length", C.c_double), ("side_length", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("steps", C.c_int64), ("bonds", C.c_int64), ("broken_bonds", C.c_int64),
                ("contact_pairs", C.c_int64), ("device_ms", C.c_double), ("newton_iterations", C.c_int64),
                ("cg_iterations", C.c_int64), ("final_residual", C.c_double),
                ("preconditioner_fallbacks", C.c_int64), ("coarse_builds", C.c_int64)]


PD_PRECOND_NONE = 0
PD_PRECOND_BLOCK_JACOBI = 1
PD_PRECOND_MPNN = 2
PD_PRECOND_TWO_LEVEL = 3


class QsOptions(C.Structure):
    _fields_ = [("newton_tolerance", C.c_double), ("cg_relative_tolerance", C.c_double),
                ("max_newton_iterations", C.c_int32), ("max_cg_iterations", C.c_int32),
                ("preconditioner", C.c_int32), ("use_predictor", C.c_int32), ("coarse_cell", C.c_double)]


class ImplicitOptions(C.Structure):
    _fields_ = [("beta", C.c_double), ("gamma", C.c_double), ("absolute_tolerance", C.c_double),
                ("cg_relative_tolerance", C.c_double), ("max_newton_iterations", C.c_int32),
                ("max_cg_iterations", C.c_int32), ("preconditioner", C.c_int32)]


# name -> (restype, argtypes); every symbol include/pd_b200.h declares.
SIGNATURES = {
    "pd_create": (C.c_int, [C.POINTER(Config), C.POINTER(_vp)]),
    "pd_destroy": (C.c_int, [_vp]),
    "pd_last_error": (C.c_char_p, [_vp]),
    "pd_version": (C.c_char_p, []),
    "pd_set_points": (C.c_int, [_vp, C.c_int64, _dp, _dp, _i32p]),
    "pd_set_block_horizons": (C.c_int, [_vp, C.c_int32, _dp]),
    "pd_build_bonds": (C.c_int, [_vp, C.POINTER(PlaneFilter), C.c_int32]),
    "pd_set_bonds": (C.c_int, [_vp, _i32p, C.c_int64]),
    "pd_num_bonds": (C.c_int, [_vp, _i64p]),
    "pd_get_bonds": (C.c_int, [_vp, _i32p, C.c_int64, _i64p]),
    "pd_material_lps": (C.c_int, [_vp, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "pd_material_lps_field": (C.c_int, [_vp, _dp, _dp]),
    "pd_material_bond_based": (C.c_int, [_vp, C.c_int32, C.c_double, C.c_double, C.c_int32, C.c_double]),
    "pd_material_linear_lps": (C.c_int, [_vp, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "pd_damage_critical_stretch": (C.c_int, [_vp, C.c_int32, C.c_double]),
    "pd_damage_critical_stretch_field": (C.c_int, [_vp, _dp]),
    "pd_weighted_volume": (C.c_int, [_vp, _dp]),
    "pd_compute_force": (C.c_int, [_vp, _dp, _dp]),
    "pd_compute_force_device": (C.c_int, [_vp, _vp, _vp]),
    "pd_compute_damage": (C.c_int, [_vp, _dp]),
    "pd_update_state": (C.c_int, [_vp]),
    "pd_set_bond_damage": (C.c_int, [_vp, _dp]),
    "pd_critical_time_step": (C.c_int, [_vp, _dp]),
    "pd_critical_time_step_static": (C.c_int, [_vp, _dp]),
    "pd_verlet_begin": (C.c_int, [_vp, C.c_double, C.c_double]),
    "pd_verlet_step": (C.c_int, [_vp, C.c_int64]),
    "pd_verlet_finish": (C.c_int, [_vp, C.POINTER(Stats)]),
    "pd_pack_state_device": (C.c_int, [_vp, C.c_int64, _vp, _vp]),
    "pd_unpack_state_device": (C.c_int, [_vp, C.c_int64, _vp, _vp]),
    "pd_set_state": (C.c_int, [_vp, _dp, _dp]),
    "pd_add_prescribed_displacement": (C.c_int, [_vp, C.c_int64, _i64p, C.c_int32, C.c_double, C.c_double]),
    "pd_add_prescribed_displacement_function": (C.c_int, [_vp, C.c_int64, _i64p, C.c_int32, C.c_char_p]),
    "pd_expr_eval": (C.c_int, [C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double, _dp]),
    "pd_clear_boundary_conditions": (C.c_int, [_vp]),
    "pd_verlet_run": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int64, C.POINTER(Stats)]),
    "pd_get_field": (C.c_int, [_vp, C.c_int32, _dp]),
    "pd_contact_short_range": (C.c_int, [_vp, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "pd_contact_force": (C.c_int, [_vp, _dp, _dp, _dp]),
    "pd_qs_load_step": (C.c_int, [_vp, C.c_double, C.c_double, C.c_void_p, C.POINTER(Stats)]),
    "pd_qs_coarse_modes": (C.c_int, [_vp, C.c_int32]),
    "pd_implicit_run": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int64, C.c_void_p, C.POINTER(Stats)]),
    "pd_jacobian_apply": (C.c_int, [_vp, _dp, _dp, _dp]),
    "pd_jacobian_block_diagonal": (C.c_int, [_vp, _dp, _dp]),
    "pd_mpnn_init": (C.c_int, [_vp, C.c_uint64, C.c_double]),
    "pd_mpnn_collect": (C.c_int, [_vp, C.c_int32]),
    "pd_mpnn_num_pairs": (C.c_int, [_vp, _i64p]),
    "pd_mpnn_train": (C.c_int, [_vp, C.c_int32, C.c_double, C.c_int32, _dp]),
    "pd_mpnn_num_params": (C.c_int, [_i64p]),
    "pd_mpnn_get_weights": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "pd_mpnn_set_weights": (C.c_int, [_vp, C.POINTER(C.c_float)]),
    "pd_mpnn_loss_grad": (C.c_int, [_vp, C.POINTER(C.c_float), _dp, C.POINTER(C.c_float)]),
    "pd_mpnn_apply": (C.c_int, [_vp, _dp, _dp]),
    "pd_mpnn_coarse": (C.c_int, [_vp, C.c_double]),
    "pd_block_data": (C.c_int, [_vp, C.c_int32, C.c_int32, C.c_int32, _dp]),
    "pd_kinetic_energy": (C.c_int, [_vp, _dp, _dp]),
    "pd_linear_momentum": (C.c_int, [_vp, _dp, _dp]),
    "pd_qs_coarse_operator": (C.c_int, [_vp, _dp, C.c_double, _i64p, _i32p, _dp, _dp]),
    "pd_set_kernel_timing": (C.c_int, [_vp, C.c_int]),
    "pd_get_kernel_timing": (C.c_int, [_vp, _dp, _i64p]),
}

_lib = None


class PDError(RuntimeError):
    """Raised for a non-zero status from the C ABI (the reference throws or terminates)."""

    def __init__(self, code, msg):
        super().__init__(f"[pd status {code}] {msg}")
        self.code = code


def load():
    """Load libpd_b200.so and bind every declared symbol. Raises if absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with peridigm_b200.build.build() "
                               "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def extra_signature(name, restype, argtypes):
    """Bind a symbol declared in include/pd_b200.h after SIGNATURES was written."""
    SIGNATURES[name] = (restype, argtypes)
    if _lib is not None:
        fn = getattr(_lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
