"""ctypes binding of the C ABI in include/cup3d_b200.h.

The library is the in-tree cup3d_b200/libcup3d_b200.so built for sm_100a by
cup3d_b200.build.  There is no fallback: if it is missing, loading fails with
an error that says how to build it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcup3d_b200.so"

CUP_OK = 0
CUP_SOFT_MAXITER = 1
CUP_SOFT_FALLBACK = 2
CUP_ERR_CUDA = -1
CUP_ERR_ARG = -2
CUP_ERR_MESH = -3
CUP_ERR_NAN = -4
CUP_ERR_STATE = -5

CNN_FORWARD_NOALLOC_MAX = 64  # CUP_CNN_FORWARD_NOALLOC_MAX

BC = {"freespace": 0, "periodic": 1, "wall": 2}
ADV = {"upwind5": 0, "upwind3": 0, "weno5": 1}
SOLVER = {"b200": 0, "b200_mixed": 1, "b200_learned": 2, "b200_learned_mixed": 3, "b200_twolevel": 4, "b200_schwarz": 5, "b200_pipelined": 6,
          "b200_twolevel_mixed": 7}
FIELD = {"vel": 0, "pres": 1, "chi": 2, "lhs": 3, "tmpV": 4}
FIELD_NCOMP = {"vel": 3, "pres": 1, "chi": 1, "lhs": 1, "tmpV": 3}


class cup_config(C.Structure):
    _fields_ = [
        ("bpd", C.c_int32 * 3),
        ("level_max", C.c_int32),
        ("bc", C.c_int32 * 3),
        ("extent", C.c_double),
        ("nu", C.c_double),
        ("cfl", C.c_double),
        ("rampup", C.c_int32),
        ("lambda_", C.c_double),
        ("implicit_penalization", C.c_int32),
        ("uinf", C.c_double * 3),
        ("advection", C.c_int32),
        ("mean_constraint", C.c_int32),
        ("poisson_tol", C.c_double),
        ("poisson_tol_rel", C.c_double),
        ("poisson_solver", C.c_int32),
        ("poisson_max_iter", C.c_int32),
        ("poisson_max_restarts", C.c_int32),
        ("step_2nd_start", C.c_int32),
        ("device", C.c_int32),
        ("poisson_block_cache", C.c_int32),
        ("step_graph", C.c_int32),
        ("static_obstacles", C.c_int32),
        ("rtol", C.c_double),
        ("ctol", C.c_double),
        ("level_max_vorticity", C.c_int32),
        ("level_start", C.c_int32),
        ("poisson_persistent", C.c_int32),
    ]


class cup_solve_stats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("restarts", C.c_int32),
        ("status", C.c_int32),
        ("fallback", C.c_int32),
        ("err_init", C.c_double),
        ("err_final", C.c_double),
        ("true_rel", C.c_double),
        ("milliseconds", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# name -> (restype, argtypes); every symbol of include/cup3d_b200.h
_P = C.c_void_p
_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int32)
SIGNATURES = {
    "cup_config_default": (None, [C.POINTER(cup_config)]),
    "cup_config_parse": (C.c_int, [C.POINTER(cup_config), C.c_char_p]),
    "cup_create": (_P, [C.POINTER(cup_config)]),
    "cup_destroy": (None, [_P]),
    "cup_last_error": (C.c_char_p, [_P]),
    "cup_set_mesh": (C.c_int, [_P, C.c_int32, _I, _I]),
    "cup_set_mesh_uniform": (C.c_int, [_P]),
    "cup_set_mesh_sphere_wake": (C.c_int, [_P, _D, C.c_double, C.c_int32, C.c_double, C.c_double, C.c_double]),
    "cup_set_mesh_random": (C.c_int, [_P, C.c_uint64, C.c_double]),
    "cup_num_blocks": (C.c_int32, [_P]),
    "cup_get_blocks": (C.c_int, [_P, _I, _I, _D]),
    "cup_get_faces": (C.c_int, [_P, _I, _I]),
    "cup_upload_field": (C.c_int, [_P, C.c_int32, _D]),
    "cup_download_field": (C.c_int, [_P, C.c_int32, _D]),
    "cup_upload_field_blocks": (C.c_int, [_P, C.c_int32, C.c_int32, _I, _I, C.POINTER(_D)]),
    "cup_download_field_blocks": (C.c_int, [_P, C.c_int32, C.c_int32, _I, _I, C.POINTER(_D)]),
    "cup_field_device_ptr": (C.c_void_p, [_P, C.c_int32]),
    "cup_stream": (C.c_void_p, [_P]),
    "cup_poisson_apply_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.c_int32]),
    "cup_block_inverse_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "cup_poisson_solve_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.POINTER(cup_solve_stats)]),
    "cup_poisson_solve": (C.c_int, [_P, C.POINTER(cup_solve_stats)]),
    "cup_batch_create": (_P, [C.c_int32, C.POINTER(_P)]),
    "cup_batch_num_cases": (C.c_int32, [_P]),
    "cup_batch_case_blocks": (C.c_int, [_P, C.c_int32, _I, _I]),
    "cup_batch_poisson_solve_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p, C.POINTER(cup_solve_stats)]),
    "cup_batch_step": (C.c_int, [_P, C.c_int32, _D, _D, _D, C.POINTER(cup_solve_stats)]),
    "cup_autotune": (C.c_int, [_P, _I, C.POINTER(C.c_float)]),
    "cup_obstacle_sphere": (C.c_int, [_P, _D, C.c_double, _D, _D]),
    "cup_obstacle_ellipsoid": (C.c_int, [_P, _D, _D, _D, _D, _D]),
    "cup_obstacle_sphere_dev": (C.c_int, [_P, _D, C.c_double, _D, _D]),
    "cup_obstacle_ellipsoid_dev": (C.c_int, [_P, _D, _D, _D, _D, _D]),
    "cup_obstacle_free": (C.c_int, [_P, _I, _I]),
    "cup_update_obstacles": (C.c_int, [_P, C.c_double, _D]),
    "cup_create_obstacles": (C.c_int, [_P, C.c_double, C.c_int32]),
    "cup_obstacle_fix_frame": (C.c_int, [_P, _I]),
    "cup_get_uinf": (C.c_int, [_P, _D]),
    "cup_compute_dissipation": (C.c_int, [_P, _D]),
    "cup_write_restart": (C.c_int, [_P, C.c_char_p, C.c_int32, C.c_double]),
    "cup_read_restart": (C.c_int, [_P, C.c_char_p, C.c_int32, _D]),
    "cup_set_obstacle": (C.c_int, [_P, C.c_int32, _I, _D, _D, _D]),
    "cup_get_obstacle": (C.c_int, [_P, _I, _D, _D, _D]),
    "cup_max_u": (C.c_int, [_P, _D]),
    "cup_compute_dt": (C.c_int, [_P, C.c_int32, _D]),
    "cup_advect_diffuse": (C.c_int, [_P, C.c_double]),
    "cup_penalize": (C.c_int, [_P, C.c_double, _D]),
    "cup_pressure_project": (C.c_int, [_P, C.c_double, C.c_int32, C.POINTER(cup_solve_stats)]),
    "cup_step": (C.c_int, [_P, C.c_int32, C.c_double, _D, C.POINTER(cup_solve_stats)]),
    "cup_pressure_rhs": (C.c_int, [_P, C.c_double, C.c_int32]),
    "cup_pressure_finish": (C.c_int, [_P, C.c_double, C.c_int32]),
    "cup_set_barrier_limit": (C.c_int, [_P, C.c_int64]),
    "cup_adapt_indicator": (C.c_int, [_P, _D]),
    "cup_adapt_mesh": (C.c_int, [_P, C.POINTER(C.c_int32)]),
    "cup_coarse_matrix": (C.c_int, [_P, _D, C.POINTER(C.c_int32)]),
    "cup_cnn_holdout": (C.c_int, [_P, C.c_int32]),
    "cup_cnn_eval": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "cup_coarse_apply_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "cup_dense_inverse_dev": (C.c_int, [_P, C.c_void_p, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    "cup_set_poisson": (C.c_int, [_P, C.c_int32, C.c_double, C.c_double, C.c_int32]),
    "cup_cnn_num_params": (C.c_int32, []),
    "cup_cnn_init": (C.c_int, [_P, C.c_uint64]),
    "cup_cnn_set_params": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "cup_cnn_get_params": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "cup_cnn_dataset_reserve": (C.c_int, [_P, C.c_int32]),
    "cup_cnn_dataset_add": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "cup_cnn_dataset_size": (C.c_int32, [_P]),
    "cup_cnn_train": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_float, C.c_uint64, C.POINTER(C.c_float)]),
    "cup_cnn_forward_host": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32]),
    "cup_cnn_grad_host": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32,
                                    C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "cup_cnn_precond_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "cup_cnn_map_apply_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "cup_schwarz_apply_dev": (C.c_int, [_P, C.c_void_p, C.c_void_p]),
    "cup_compute_forces": (C.c_int, [_P, _D]),
    "cup_cnn_forward_host_noalloc": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int32]),
    "cup_profile": (C.c_int, [_P, C.c_int32]),
    "cup_profile_read": (C.c_int, [_P, C.c_char_p, C.c_int32]),
}


def lib():
    """Loads libcup3d_b200.so (once) and declares every C-ABI signature."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m cup3d_b200.build` "
                "(there is no CPU fallback for the hot path)")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class CupError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"cup3d_b200 error {code}: {msg}")
        self.code = code


def check(rc, ctx=None):
    if rc < 0:
        msg = lib().cup_last_error(ctx)
        raise CupError(rc, msg.decode() if msg else "")
    return rc


def dptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_D)


def iptr(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(_I)
