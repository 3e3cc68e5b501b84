"""ctypes binding of libpigfem_b200.so (the C ABI in include/pigfem_b200.h).

The library is loaded from the package directory.  There is no CPU fallback:
if the shared object is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpigfem_b200.so")

PG_OK = 0
PG_STATIC_MAX_NODES = 32768
PG_ERR_ARG = 1
PG_ERR_MESH = 2
PG_ERR_CUDA = 3
PG_ERR_NOT_CONVERGED = 4
PG_ERR_BREAKDOWN = 5
PG_ERR_STATE = 6
PG_ERR_LIMIT = 7

PG_COH_OP = 0
PG_COH_BILINEAR = 1
PG_KRYLOV_CG = 0
PG_KRYLOV_GMRES = 1
PG_KRYLOV_MINRES = 2
PG_PREC_JACOBI = 0
PG_PREC_BLOCK_JACOBI = 1
PG_PREC_NONE = 2
PG_PREC_MG = 3
PG_RTOL_BASE_PREDICTOR = 0
PG_RTOL_BASE_ZEROTH = 1
PG_PRECISION_FP64 = 0
PG_PRECISION_MIXED = 1
PG_SHAPE_X = 0
PG_SHAPE_Y = 1
PG_SHAPE_R = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_u8p = C.POINTER(C.c_uint8)


class RveDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32),
        ("x0", C.c_double), ("x1", C.c_double), ("y0", C.c_double), ("y1", C.c_double),
        ("n_inclusions", C.c_int32),
        ("inc_cx", _dp), ("inc_cy", _dp), ("inc_r", _dp), ("inc_mat", _ip),
        ("n_materials", C.c_int32), ("mat_E", _dp), ("mat_nu", _dp),
        ("matrix_mat", C.c_int32), ("plane_strain", C.c_int32), ("cohesive", C.c_int32),
        ("coh_law", C.c_int32), ("coh_params", C.c_double * 5), ("strain", C.c_double),
    ]


class MeshInfo(C.Structure):
    _fields_ = [(n, C.c_int32) for n in (
        "n_nodes", "n_regular_nodes", "n_enrichment_nodes", "n_elements", "n_cut_elements",
        "n_cohesive_qp", "n_dof", "n_free_dof", "n_blocks", "n_moved_nodes")]


class SolverCfg(C.Structure):
    _fields_ = [
        ("krylov", C.c_int32), ("precond", C.c_int32), ("precision", C.c_int32),
        ("rtol", C.c_double), ("max_iter", C.c_int32), ("inner_rtol", C.c_double),
        ("max_refine", C.c_int32), ("gmres_restart", C.c_int32), ("check_every", C.c_int32),
        ("inclusion_modes", C.c_int32), ("deterministic", C.c_int32),
    ]


class SolveStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32), ("refinements", C.c_int32), ("rel_residual", C.c_double),
        ("seconds", C.c_double), ("newton_iterations", C.c_int32), ("status", C.c_int32),
    ]


PG_PREDICT_ZEROTH = 0
PG_PREDICT_LINEAR = 1
PG_PREDICT_GIVEN = 2
PG_PREDICT_LEARNED = 3


class NewtonCfg(C.Structure):
    _fields_ = [
        ("n_steps", C.c_int32), ("T_final", C.c_double), ("rtol", C.c_double), ("atol", C.c_double),
        ("stol", C.c_double), ("max_it", C.c_int32), ("precision", C.c_int32), ("precond", C.c_int32),
        ("lin_rtol", C.c_double), ("inner_rtol", C.c_double), ("lin_max_iter", C.c_int32),
        ("max_repeat", C.c_int32), ("predictor", C.c_int32), ("rtol_base", C.c_int32),
        ("inclusion_modes", C.c_int32), ("t_start", C.c_double), ("t_stop", C.c_double),
        ("deterministic", C.c_int32),
    ]


class StepStats(C.Structure):
    _fields_ = [
        ("t_frac", C.c_double), ("dt", C.c_double), ("newton_its", C.c_int32), ("krylov_its", C.c_int32),
        ("gmres_fallbacks", C.c_int32), ("repeats", C.c_int32), ("res0", C.c_double), ("res", C.c_double),
        ("reason", C.c_int32), ("seconds", C.c_double), ("predictor_used", C.c_int32),
        ("res_linear", C.c_double), ("res_learned", C.c_double), ("res_base", C.c_double), ("blend", C.c_double),
    ]


class PredHistory(C.Structure):
    """pg_pred_history: device pointers of the last three converged states
    and of the committed delta_max one step back, the step lengths, the load
    fraction and the prescribed increment of the coming step."""
    _fields_ = [("U_n", C.c_void_p), ("U_nm1", C.c_void_p), ("U_nm2", C.c_void_p), ("isv_nm1", C.c_void_p),
                ("dt_n", C.c_double), ("dt_nm1", C.c_double), ("dt", C.c_double), ("t_frac", C.c_double),
                ("s_inc", C.c_double)]


class PgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[pg status {code}] {msg}")
        self.code = code


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m pigfem_assignment_b200.build` "
            "(this package has no CPU fallback)")
    lib = C.CDLL(LIB_PATH)
    v = C.c_void_p
    sig = {
        "pg_mesh_build": ([C.POINTER(RveDesc), C.POINTER(v)], C.c_int),
        "pg_mesh_build_device": ([C.POINTER(RveDesc), C.c_int32, C.POINTER(v)], C.c_int),
        "pg_mesh_info_get": ([v, C.POINTER(MeshInfo)], C.c_int),
        "pg_mesh_export": ([v, _dp, _ip, _ip, _ip, _ip, _u8p, _dp], C.c_int),
        "pg_mesh_export_cut": ([v, _ip, _ip, _ip, _ip, _ip], C.c_int),
        "pg_mesh_export_pattern": ([v, _ip, _ip], C.c_int),
        "pg_template_table": ([_ip, _ip], C.c_int),
        "pg_mesh_destroy": ([v], None),
        "pg_ctx_create": ([v, C.c_int32, C.POINTER(v)], C.c_int),
        "pg_ctx_destroy": ([v], None),
        "pg_ctx_sync": ([v], C.c_int),
        "pg_assemble_linear": ([v, v], C.c_int),
        "pg_assemble_linear_host": ([v, _dp, _dp], C.c_int),
        "pg_assemble_nonlinear": ([v, _dp, C.c_double, C.c_int32, C.c_int32, v], C.c_int),
        "pg_new_load_step": ([v, C.c_double], C.c_int),
        "pg_stress_strain": ([v, _dp, _dp, C.POINTER(C.c_int64), _ip, _dp], C.c_int),
        "pg_write_vtk": ([v, C.c_char_p, C.c_double], C.c_int),
        "pg_write_cohesive_openings": ([v, C.c_char_p], C.c_int),
        "pg_commit_isv": ([v], C.c_int),
        "pg_ctx_device_arrays": ([v, C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp),
                                  C.POINTER(_dp)], C.c_int),
        "pg_solver_cfg_default": ([C.POINTER(SolverCfg)], None),
        "pg_solve_linear": ([v, C.POINTER(SolverCfg), C.POINTER(SolveStats)], C.c_int),
        "pg_sensitivity_c11": ([v, C.POINTER(SolverCfg), C.c_double, _dp, _dp, C.POINTER(SolveStats)], C.c_int),
        "pg_sensitivity_shape": ([v, C.POINTER(SolverCfg), C.c_int32, _ip, _ip, _dp, _dp, C.POINTER(SolveStats)],
                                 C.c_int),
        "pg_ctx_autotune": ([v, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
        "pg_ctx_tuning": ([v, _ip, _ip, _ip], C.c_int),
        "pg_ctx_set_tuning": ([v, C.c_int32, C.c_int32, C.c_int32], C.c_int),
        "pg_ctx_cut_overlap": ([v, C.c_int32, _ip], C.c_int),
        "pg_batch_create": ([C.POINTER(C.c_void_p), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)], C.c_int),
        "pg_batch_destroy": ([v], None),
        "pg_batch_context": ([v], C.c_void_p),
        "pg_batch_setup_times": ([v, C.POINTER(C.c_double)], C.c_int),
        "pg_batch_info": ([v, _ip, _ip, _ip], C.c_int),
        "pg_batch_solve": ([v, C.POINTER(SolverCfg), C.POINTER(SolveStats), C.POINTER(SolveStats)], C.c_int),
        "pg_batch_get_solution": ([v, C.c_int32, _dp], C.c_int),
        "pg_pcg_solve_static": ([C.c_int32, v, v, v, v, v, v, C.c_double, C.c_int32, v, C.POINTER(SolveStats)],
                                C.c_int),
        "pg_get_matrix": ([v, _dp], C.c_int),
        "pg_get_vector": ([v, C.c_int32, _dp], C.c_int),
        "pg_set_vector": ([v, C.c_int32, _dp], C.c_int),
        "pg_get_isv": ([v, C.c_int32, _dp], C.c_int),
        "pg_set_isv": ([v, C.c_int32, _dp], C.c_int),
        "pg_assembly_timing": ([v, C.c_int32, C.POINTER(C.c_float), C.POINTER(C.c_float)], C.c_int),
        "pg_newton_cfg_default": ([C.POINTER(NewtonCfg)], None),
        "pg_newton_load_step": ([v, C.c_double, C.c_double, C.POINTER(NewtonCfg), C.POINTER(StepStats)], C.c_int),
        "pg_solve_nonlinear": ([v, C.POINTER(NewtonCfg), C.POINTER(StepStats), C.c_int32, C.POINTER(C.c_int32)],
                               C.c_int),
        "pg_mlp_create": ([C.c_int32, C.c_uint64, C.POINTER(v)], C.c_int),
        "pg_mlp_destroy": ([v], None),
        "pg_mlp_param_count": ([], C.c_int32),
        "pg_mlp_params": ([v, C.POINTER(C.c_float), C.c_int32], C.c_int),
        "pg_mlp_grads": ([v, C.POINTER(C.c_float)], C.c_int),
        "pg_mlp_forward": ([v, v, C.c_int32, v, v], C.c_int),
        "pg_mlp_gradient": ([v, v, v, C.c_int32, C.POINTER(C.c_double)], C.c_int),
        "pg_mlp_adam": ([v, C.c_float], C.c_int),
        "pg_mlp_train": ([v, v, v, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.POINTER(C.c_double)], C.c_int),
        "pg_mlp_wait_selftest": ([v, C.c_int32], C.c_int),
        "pg_predictor_features": ([v, C.POINTER(PredHistory), v], C.c_int),
        "pg_predictor_targets": ([v, C.POINTER(PredHistory), v, v], C.c_int),
        "pg_predictor_apply": ([v, C.POINTER(PredHistory), v, C.c_double, v], C.c_int),
        "pg_ctx_attach_mlp": ([v, v], C.c_int),
        "pg_last_error": ([], C.c_char_p),
        "pg_version": ([], C.c_char_p),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    return lib


lib = _load()

# every extern "C" symbol include/pigfem_b200.h declares
DECLARED_SYMBOLS = (
    "pg_mesh_build", "pg_mesh_build_device", "pg_mesh_info_get", "pg_mesh_export", "pg_mesh_export_cut", "pg_mesh_export_pattern",
    "pg_template_table", "pg_mesh_destroy", "pg_ctx_create", "pg_ctx_destroy", "pg_ctx_sync",
    "pg_assemble_linear", "pg_assemble_linear_host", "pg_assemble_nonlinear", "pg_stress_strain", "pg_write_vtk", "pg_write_cohesive_openings", "pg_new_load_step",
    "pg_commit_isv", "pg_ctx_device_arrays", "pg_solver_cfg_default", "pg_solve_linear", "pg_get_matrix",
    "pg_get_vector", "pg_set_vector", "pg_get_isv", "pg_set_isv", "pg_assembly_timing", "pg_newton_cfg_default", "pg_newton_load_step",
    "pg_solve_nonlinear", "pg_mlp_create", "pg_mlp_destroy", "pg_mlp_param_count", "pg_mlp_params",
    "pg_mlp_grads", "pg_mlp_forward", "pg_mlp_gradient", "pg_mlp_adam", "pg_mlp_train", "pg_mlp_wait_selftest", "pg_predictor_features",
    "pg_predictor_targets", "pg_predictor_apply", "pg_ctx_attach_mlp", "pg_sensitivity_c11", "pg_sensitivity_shape", "pg_ctx_autotune", "pg_ctx_tuning", "pg_ctx_set_tuning", "pg_ctx_cut_overlap", "pg_batch_create", "pg_batch_destroy", "pg_batch_context", "pg_batch_setup_times",
    "pg_batch_info", "pg_batch_solve", "pg_batch_get_solution", "pg_pcg_solve_static", "pg_last_error",
    "pg_version",
)


def check(rc: int, what: str = "") -> None:
    if rc != PG_OK:
        msg = lib.pg_last_error()
        raise PgError(rc, (what + ": " if what else "") + (msg.decode() if msg else ""))


def dptr(a):
    return a.ctypes.data_as(_dp)


def iptr(a):
    return a.ctypes.data_as(_ip)


def u8ptr(a):
    return a.ctypes.data_as(_u8p)
