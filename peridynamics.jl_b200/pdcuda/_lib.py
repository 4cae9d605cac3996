"""ctypes binding of libpdcuda (the C ABI declared in include/pdcuda.h).

The library is loaded from this package directory. There is no CPU fallback: when the
library is missing or the machine has no CUDA device, the calls fail with an error.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpdcuda.so")
_LIB = None

# status codes
(PD_OK, PD_ERR_ARG, PD_ERR_CUDA, PD_ERR_NAN, PD_ERR_TIMEOUT, PD_ERR_OOM, PD_ERR_UNSUPPORTED,
 PD_ERR_NOCONV) = range(8)
# materials, models, kernels, precision
MAT_BB, MAT_OSB, MAT_CMAT = 0, 1, 2
CM_SVK, CM_NEOHOOKE, CM_NEOHOOKE_PENALTY = 0, 1, 2
ZEM_SILLING, ZEM_WAN = 0, 1
KERNEL_CONST_ONE, KERNEL_LINEAR, KERNEL_CUBIC_BSPLINE = 0, 1, 2
PREC_FP64, PREC_FP32_KAHAN = 0, 1
# fields
(F_POSITION, F_DISPLACEMENT, F_VELOCITY, F_VELOCITY_HALF, F_ACCELERATION, F_B_INT, F_B_EXT,
 F_DAMAGE, F_N_ACTIVE_BONDS, F_BOND_ACTIVE, F_DEFGRAD, F_CAUCHY_STRESS, F_N_NEIGHBORS) = range(13)
BC_VELOCITY_HALF, BC_B_EXT = 0, 1
BC_KIND_TIME, BC_KIND_POINT_TIME, BC_KIND_DATA = 0, 1, 2
# Newton-Krylov: Frechet rules, preconditioners, condition fields
NK_CENTRAL, NK_FORWARD = 0, 1
PC_NONE, PC_BLOCK_JACOBI, PC_BLOCK_POLY, PC_LEARNED_POLY, PC_LEARNED = range(5)
NKC_DISPLACEMENT, NKC_B_EXT = 0, 1
MPNN_N_PARAMS = 18185

# every symbol that include/pdcuda.h declares
EXPORTS = (
    "pd_last_error", "pd_version", "pd_find_bonds", "pd_create", "pd_create_search",
    "pd_destroy", "pd_set_state", "pd_break_bonds", "pd_break_random_pairs", "pd_get_field",
    "pd_set_bcs", "pd_set_bc_values", "pd_stable_timestep", "pd_set_param_timesteps",
    "pd_force", "pd_run_vv", "pd_nan_step", "pd_run_vv_timed", "pd_autotune", "pd_set_mapping",
    "pd_set_graph", "pd_set_pipeline", "pd_get_mapping", "pd_info", "pd_launch_count", "pd_stream",
    "pd_dr_init", "pd_run_dr", "pd_run_dr_timed", "pd_dr_density_matrix",
    "pd_break_random_pairs_ids", "pd_create_partition", "pd_set_stream", "pd_vv_begin",
    "pd_force_phase", "pd_vv_stage", "pd_vv_end", "pd_halo_row_bytes", "pd_halo_pack",
    "pd_halo_unpack", "pd_esc_init", "pd_esc_get", "pd_count_near_critical",
    "pd_nk_set_conditions", "pd_nk_step", "pd_nk_set_corrections", "pd_nk_apply",
    "pd_nk_record", "pd_nk_recorded", "pd_nk_recorded_vector",
    "pd_mpnn_create", "pd_mpnn_destroy", "pd_mpnn_set_params", "pd_mpnn_get_params",
    "pd_mpnn_infer", "pd_mpnn_loss_grad", "pd_mpnn_spectral_grad", "pd_mpnn_zero_grad",
    "pd_mpnn_adam",
    "pd_osb_force_static", "pd_static_last_error",
    "pd_group_create", "pd_group_run_vv", "pd_group_destroy",
)


class PointParams(C.Structure):
    _fields_ = [(k, C.c_double) for k in
                ("delta", "rho", "E", "nu", "G", "K", "lambda_", "mu", "Gc", "epsilon_c", "bc")]


class BodyDesc(C.Structure):
    _fields_ = [("n_points", C.c_int64), ("position", C.c_void_p), ("volume", C.c_void_p),
                ("n_bonds", C.c_int64), ("bond_offsets", C.c_void_p), ("neighbors", C.c_void_p),
                ("bond_length", C.c_void_p), ("fail_permit", C.c_void_p),
                ("param_id", C.c_void_p), ("n_params", C.c_int32), ("params", C.c_void_p),
                ("material", C.c_int32), ("kernel", C.c_int32), ("cmodel", C.c_int32),
                ("precision", C.c_int32), ("multi_params", C.c_int32), ("zem_cs", C.c_double),
                ("maxdmg", C.c_double), ("device", C.c_int32), ("zem", C.c_int32)]


class BCDesc(C.Structure):
    _fields_ = [("field", C.c_int32), ("dim", C.c_int32), ("kind", C.c_int32),
                ("n_points", C.c_int32), ("points", C.c_void_p), ("data", C.c_void_p)]


class NKCondition(C.Structure):
    _fields_ = [("field", C.c_int32), ("dim", C.c_int32), ("n_points", C.c_int64),
                ("points", C.c_void_p), ("values", C.c_void_p)]


class NKParams(C.Structure):
    _fields_ = [("maxiter", C.c_int32), ("tol", C.c_double), ("tol_relative", C.c_int32),
                ("perturbation_scale", C.c_double), ("frechet", C.c_int32),
                ("gmres_maxiter", C.c_int32), ("gmres_reltol", C.c_double),
                ("gmres_abstol", C.c_double), ("gmres_restart", C.c_int32),
                ("precond", C.c_int32)]


class NKStats(C.Structure):
    _fields_ = [("newton_iters", C.c_int32), ("converged", C.c_int32),
                ("gmres_iters", C.c_int64), ("matvecs", C.c_int64),
                ("force_evals", C.c_int64), ("precond_applies", C.c_int64),
                ("residual_first", C.c_double), ("residual", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class NaNError(RuntimeError):
    """NaN values in the internal force density (the reference's NaNError, errors.jl:98-114)."""

    def __init__(self, time, step):
        self.time = time
        self.step = step
        super().__init__(f"NaN values detected in force density field!\n  time:    {time}\n"
                         f"  step:    {step}")


class PDCudaError(RuntimeError):
    pass


class NotConvergedError(RuntimeError):
    """Newton iterations exhausted (the reference's ErrorException, newton_krylov.jl:317-324)."""


def lib():
    """Load libpdcuda.so. Fails loudly when it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise PDCudaError(f"libpdcuda.so not built ({LIB_PATH}); run __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    vp, i64, i32, dbl, st = C.c_void_p, C.c_int64, C.c_int32, C.c_double, C.c_int32
    L.pd_last_error.restype = C.c_char_p
    L.pd_version.restype = C.c_char_p
    L.pd_static_last_error.restype = C.c_char_p
    sig = {
        "pd_find_bonds": [i64, vp, vp, vp, i32, vp, vp, i64, vp, vp, vp, vp, vp, i32],
        "pd_create": [vp, vp],
        "pd_create_search": [vp, vp, vp, i32, vp, vp, vp],
        "pd_destroy": [vp],
        "pd_set_state": [vp, vp, vp, vp, vp, vp, vp, vp],
        "pd_break_bonds": [vp, vp, vp],
        "pd_break_random_pairs": [vp, dbl, C.c_uint64],
        "pd_get_field": [vp, i32, vp, C.c_size_t],
        "pd_set_bcs": [vp, i32, vp],
        "pd_set_bc_values": [vp, i64, i64, vp, i64],
        "pd_stable_timestep": [vp, dbl, vp, vp],
        "pd_set_param_timesteps": [vp, vp],
        "pd_force": [vp, dbl, dbl],
        "pd_run_vv": [vp, i64, i64, dbl],
        "pd_nan_step": [vp, vp],
        "pd_run_vv_timed": [vp, i64, i64, dbl, vp, vp, vp, vp],
        "pd_autotune": [vp, vp, vp],
        "pd_set_mapping": [vp, i32, i32],
        "pd_set_graph": [vp, i32],
        "pd_set_pipeline": [vp, i32],
        "pd_get_mapping": [vp, vp, vp, vp],
        "pd_info": [vp, vp, vp, vp],
        "pd_launch_count": [vp, vp],
        "pd_stream": [vp, vp],
        "pd_osb_force_static": [i64] + [vp] * 8 + [vp, i32, vp, vp, vp],
        "pd_dr_init": [vp, dbl, dbl],
        "pd_break_random_pairs_ids": [vp, dbl, C.c_uint64, vp],
        "pd_create_partition": [vp, vp, vp, i32, vp, vp, vp, vp],
        "pd_set_stream": [vp, vp],
        "pd_vv_begin": [vp, i64, i64, dbl],
        "pd_force_phase": [vp, i32, dbl, dbl],
        "pd_vv_stage": [vp, i32, i64],
        "pd_vv_end": [vp],
        "pd_halo_row_bytes": [vp, i32, vp],
        "pd_halo_pack": [vp, i32, vp, i64, vp],
        "pd_halo_unpack": [vp, i32, vp, i64, vp],
        "pd_esc_init": [vp, i32],
        "pd_esc_get": [vp, vp, vp],
        "pd_count_near_critical": [vp, dbl, vp],
        "pd_run_dr": [vp, i64, i64],
        "pd_run_dr_timed": [vp, i64, i64, vp, vp, vp, vp],
        "pd_dr_density_matrix": [vp, vp],
        "pd_nk_set_conditions": [vp, i32, vp],
        "pd_nk_step": [vp, i64, dbl, vp, vp],
        "pd_nk_set_corrections": [vp, vp],
        "pd_nk_apply": [vp, i32, vp, vp, vp],
        "pd_nk_record": [vp, i64],
        "pd_nk_recorded": [vp, vp],
        "pd_nk_recorded_vector": [vp, i64, vp],
        "pd_mpnn_create": [i32, vp],
        "pd_mpnn_destroy": [vp],
        "pd_mpnn_set_params": [vp, vp],
        "pd_mpnn_get_params": [vp, vp],
        "pd_mpnn_infer": [vp, vp, vp, vp],
        "pd_mpnn_loss_grad": [vp, vp, i32, vp, i32, vp, dbl, dbl, vp, vp],
        "pd_mpnn_spectral_grad": [vp, vp, i32, vp, i32, vp, dbl, dbl, vp, vp],
        "pd_mpnn_zero_grad": [vp],
        "pd_mpnn_adam": [vp, C.c_float],
        "pd_group_create": [vp, i32, vp],
        "pd_group_run_vv": [vp, i64, i64, dbl, i32, vp],
        "pd_group_destroy": [vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = st
    _LIB = L
    return L


def last_error():
    return lib().pd_last_error().decode()


def check(status, what=""):
    """Map a pd_status to the reference's exception types."""
    if status == PD_OK:
        return
    msg = last_error()
    if status in (PD_ERR_ARG, PD_ERR_UNSUPPORTED):
        raise ValueError(f"{what}: {msg}" if what else msg)
    if status == PD_ERR_NAN:
        raise NaNError(None, None)
    if status == PD_ERR_NOCONV:
        raise NotConvergedError(msg)
    raise PDCudaError(f"{what}: {msg} (status {status})" if what else f"{msg} (status {status})")


def ptr(a):
    return None if a is None else a.ctypes.data
