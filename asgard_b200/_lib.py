"""ctypes binding of the C ABI in ``include/asgard_b200.h``.

Loads the in-tree ``libasgard_b200.so``.  There is no fallback: if the library
is missing or does not load, importing fails with the reason.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libasgard_b200.so")

EXPORTS = [
    "asgk_plan_create", "asgk_plan_create_pairs", "asgk_plan_create_conn",
    "asgk_plan_create_global", "asgk_plan_create_dense", "asgk_plan_kind",
    "asgk_plan_update_terms", "asgk_plan_set_workspace", "asgk_plan_create_grid",
    "asgk_plan_destroy", "asgk_plan_update_values", "asgk_plan_info",
    "asgk_apply", "asgk_apply_f32", "asgk_apply_host", "asgk_apply_euler",
    "asgk_gmres_euler", "asgk_gmres_dense", "asgk_gmres_dense_precond",
    "asgk_default_gmres_restarts",
    "asgk_cgs_step", "asgk_cgs_step_noalloc",
    "asgk_sparse_grid", "asgk_connect_1d", "asgk_build_pairs",
    "asgk_direction_pairs",
    "asgk_status_string", "asgk_launch_count", "asgk_device_info",
    "asgk_device_status",
    "asgk_measure_fma_peak", "asgk_mlp_create", "asgk_mlp_destroy",
    "asgk_mlp_num_params", "asgk_mlp_get_params", "asgk_mlp_set_params",
    "asgk_mlp_forward_backward", "asgk_mlp_train", "asgk_mlp_apply",
    "asgk_mlp_train_residual", "asgk_jacobi_create", "asgk_jacobi_destroy",
    "asgk_jacobi_apply", "asgk_jacobi_apply_precision", "asgk_jacobi_info",
    "asgk_gmres_euler_jacobi",
    "asgk_mlp_set_base", "asgk_implicit_advance", "asgk_set_gmres_graphs",
    "asgk_set_gmres_basis", "asgk_set_gmres_node_steps", "asgk_imex_advance",
    "asgk_set_gmres_fused_copy", "asgk_set_bf16_inner_tol",
]


class GmresInfo(C.Structure):
    _fields_ = [("error", C.c_double), ("iterations", C.c_int),
                ("status", C.c_int), ("true_relres", C.c_double),
                ("outer_steps", C.c_int), ("matvecs_low", C.c_int),
                ("matvecs_fp64", C.c_int), ("precond_calls", C.c_int),
                ("fallback", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_vp = C.c_void_p
_i = C.c_int
# asgk_imex_hook: (ctx, step, stage, event, const double *f, stream) -> status
IMEX_HOOK = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                        C.c_void_p)
_i64 = C.c_int64
_d = C.c_double


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"asgard_b200: {LIB_PATH} is missing; build it with "
            "`python asgard_b200/build.py` (nvcc, sm_100a)")
    lib = C.CDLL(LIB_PATH)
    sig = {
        "asgk_plan_create": ([C.POINTER(_vp), _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i64], _i),
        "asgk_plan_create_pairs": ([C.POINTER(_vp), _i, _i, _i, _i, _i, _i64, _vp, _vp, _vp, _vp, _i64], _i),
        "asgk_plan_create_conn": ([C.POINTER(_vp), _i, _i, _i, _i, _i, _vp, _vp, _vp, _vp, _i64], _i),
        "asgk_plan_create_global": ([C.POINTER(_vp), _i, _i, _i, _i, _vp, _i, _vp, _i64], _i),
        "asgk_plan_create_dense": ([C.POINTER(_vp), _i, _i, _i, _i, _i, _vp, _vp, _i64, _i, _i, _i], _i),
        "asgk_plan_kind": ([_vp], _i),
        "asgk_plan_create_grid": ([C.POINTER(_vp), _i, _i, _i, _i, _vp, _i64], _i),
        "asgk_plan_set_workspace": ([_vp, _vp, _i64, _vp, _i64], _i),
        "asgk_plan_update_terms": ([_vp, _vp, _i], _i),
        "asgk_plan_destroy": ([_vp], None),
        "asgk_plan_update_values": ([_vp, _vp, _i64], _i),
        "asgk_plan_info": ([_vp] + [C.POINTER(_i64)] * 5, _i),
        "asgk_apply": ([_vp, _i, _d, _vp, _d, _vp, _vp], _i),
        "asgk_apply_f32": ([_vp, C.c_float, _vp, C.c_float, _vp, _vp], _i),
        "asgk_apply_host": ([_vp, _d, _vp, _d, _vp, _vp], _i),
        "asgk_apply_euler": ([_vp, _i, _d, _d, _vp, _d, _vp, _vp], _i),
        "asgk_gmres_euler": ([_vp, _d, _vp, _vp, _i, _i, _d, _i, _i, _vp, C.POINTER(GmresInfo), _vp], _i),
        "asgk_gmres_dense": ([_i, _vp, _vp, _vp, _i, _i, _d, C.POINTER(GmresInfo)], _i),
        "asgk_gmres_dense_precond": ([_i, _vp, _vp, _vp, _vp, _i, _i, _d,
                                      C.POINTER(GmresInfo)], _i),
        "asgk_default_gmres_restarts": ([_i64], _i),
        "asgk_cgs_step": ([_vp, _i64, _i, _vp, _i64, _vp, C.POINTER(_d), _vp], _i),
        "asgk_cgs_step_noalloc": ([_vp, _i64, _i, _vp, _i64, _vp, C.POINTER(_d), _vp], _i),
        "asgk_sparse_grid": ([_i, _i, _vp], _i64),
        "asgk_connect_1d": ([_i, C.POINTER(_i), C.POINTER(_i), _vp, _vp], _i),
        "asgk_build_pairs": ([_i, _i, _i, _vp, C.POINTER(_i64), _vp, _vp, _vp], _i),
        "asgk_direction_pairs": ([_i, _i, _i, _vp, C.POINTER(_i64), _vp, _vp, _vp, _vp], _i),
        "asgk_status_string": ([_i], C.c_char_p),
        "asgk_launch_count": ([], _i64),
        "asgk_device_info": ([C.POINTER(_i)] * 3, _i),
        "asgk_device_status": ([_i], _i),
        "asgk_measure_fma_peak": ([_i, C.POINTER(_d)], _i),
        "asgk_mlp_create": ([C.POINTER(_vp), _i, _i, _i, _vp, _i, _i, C.c_uint64], _i),
        "asgk_mlp_destroy": ([_vp], None),
        "asgk_mlp_num_params": ([_vp, C.POINTER(_i64)], _i),
        "asgk_mlp_get_params": ([_vp, _vp], _i),
        "asgk_mlp_set_params": ([_vp, _vp], _i),
        "asgk_mlp_forward_backward": ([_vp, _i, _vp, _vp, _vp, _vp, C.POINTER(_d)], _i),
        "asgk_mlp_train": ([_vp, _vp, _vp, _i, _i, _i, C.c_float, C.c_uint64, C.POINTER(_d), _vp], _i),
        "asgk_mlp_apply": ([_vp, _vp, _vp, _vp, _vp], _i),
        "asgk_jacobi_create": ([C.POINTER(_vp), _vp, _d, _i], _i),
        "asgk_jacobi_destroy": ([_vp], None),
        "asgk_mlp_set_base": ([_vp, _vp], _i),
        "asgk_jacobi_apply": ([_vp, _vp, _vp, _vp], _i),
        "asgk_jacobi_apply_precision": ([_vp, _i, _vp, _vp, _vp], _i),
        "asgk_jacobi_info": ([_vp, C.POINTER(_i), C.POINTER(_d), C.POINTER(_i64)], _i),
        "asgk_gmres_euler_jacobi": ([_vp, _d, _vp, _vp, _i, _i, _d, _i, _i, _vp, C.POINTER(GmresInfo), _vp], _i),
        "asgk_set_gmres_graphs": ([_i], _i),
        "asgk_set_gmres_basis": ([_i], _i),
        "asgk_set_gmres_fused_copy": ([_i], _i),
        "asgk_set_bf16_inner_tol": ([_d], _d),
        "asgk_set_gmres_node_steps": ([_i], _i),
        "asgk_implicit_advance": ([_vp, _d, _vp, _i, _vp, _i64, _i, _i, _d, _i, _i, _i, _vp, C.POINTER(GmresInfo), _vp], _i),
        "asgk_imex_advance": ([_vp, _vp, _d, _vp, _i, _i, _i, _d, _i, _i, _vp, _vp, _vp, _vp,
                               _vp, C.POINTER(GmresInfo), _vp], _i),
        "asgk_mlp_train_residual": ([_vp, _vp, _vp, _d, _vp, _vp, _i, _i, C.c_float, _i, C.c_uint64, C.POINTER(_d), _vp], _i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()


class AsgkError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        msg = lib.asgk_status_string(status).decode()
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)
        self.status = status


def check(status: int, what: str = "") -> None:
    if status != 0:
        raise AsgkError(status, what)
