"""ctypes binding of the cufsp C ABI (include/cufsp.h).

The shared library is built in-tree (python -m cuda_fsp_b200.build).  There is no fallback: if the
library is missing or no CUDA device is present, calls fail loudly with CufspError.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE / "lib" / "libcufsp.so"

STATUS = {0: "CUFSP_SUCCESS", 1: "CUFSP_ERR_INVALID_ARG", 2: "CUFSP_ERR_OVERFLOW", 3: "CUFSP_ERR_ALLOC",
          4: "CUFSP_ERR_CUDA", 5: "CUFSP_ERR_NONFINITE", 6: "CUFSP_ERR_STEP_LIMIT", 7: "CUFSP_ERR_UNSUPPORTED",
          8: "CUFSP_ERR_NO_DEVICE"}

FORMAT_CSR, FORMAT_HYB, FORMAT_KRONECKER = 0, 1, 2

# C function pointer types (cufsp.h)
PROP_FACTOR_FN = C.CFUNCTYPE(C.c_double, C.c_int, C.c_int, C.c_int)
TCOEF_FN = C.CFUNCTYPE(None, C.c_double, C.POINTER(C.c_double), C.c_void_p)
MATVEC_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p)


class CufspError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        self.name = STATUS.get(status, f"status {status}")
        super().__init__(f"{where}: {self.name}" + (f" ({detail})" if detail else ""))


class ModelDesc(C.Structure):
    _fields_ = [
        ("n_species", C.c_int),
        ("n_reactions", C.c_int),
        ("fsp_bounds", C.POINTER(C.c_int)),
        ("stoich_vals", C.POINTER(C.c_int)),
        ("stoich_colidxs", C.POINTER(C.c_int)),
        ("stoich_rowptrs", C.POINTER(C.c_int)),
        ("factor_tables", C.POINTER(C.c_double)),
        ("prop_factor", PROP_FACTOR_FN),
        ("prop_device", C.c_void_p),
        ("tcoef", TCOEF_FN),
        ("tcoef_user", C.c_void_p),
    ]


class ExpvStats(C.Structure):
    _fields_ = [("n_steps", C.c_int64), ("n_reject", C.c_int64), ("n_matvec", C.c_int64),
                ("n_breakdown", C.c_int64), ("t_now", C.c_double), ("last_err", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class SolverStatus(C.Structure):
    _fields_ = [("time_index", C.c_int), ("t", C.c_double), ("fsp_error", C.c_double), ("fsp_tol_exceeded", C.c_int),
                ("krylov_steps", C.c_int64), ("matvecs", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BdfStats(C.Structure):
    _fields_ = [("t", C.c_double), ("h", C.c_double), ("last_err", C.c_double), ("order", C.c_int),
                ("pad", C.c_int), ("n_steps", C.c_int64), ("n_reject", C.c_int64), ("n_matvec", C.c_int64),
                ("n_lin_iters", C.c_int64), ("n_lin_fail", C.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class BatchDesc(C.Structure):
    _fields_ = [
        ("n_species", C.c_int),
        ("n_reactions", C.c_int),
        ("stoich_vals", C.POINTER(C.c_int)),
        ("stoich_colidxs", C.POINTER(C.c_int)),
        ("stoich_rowptrs", C.POINTER(C.c_int)),
        ("n_instances", C.c_int),
        ("fsp_bounds", C.POINTER(C.c_int)),
        ("factor_tables", C.POINTER(C.POINTER(C.c_double))),
        ("coefs", C.POINTER(C.c_double)),
    ]


class BatchStat(C.Structure):
    _fields_ = [("t", C.c_double), ("err", C.c_double), ("steps", C.c_int), ("rejects", C.c_int),
                ("matvecs", C.c_int), ("status", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class AdaptiveStatus(C.Structure):
    _fields_ = [("time_index", C.c_int), ("t", C.c_double), ("fsp_error", C.c_double), ("fsp_tol_exceeded", C.c_int),
                ("expansions", C.c_int), ("n_states", C.c_int64), ("bounds", C.c_int * 16)]

    def as_dict(self) -> dict:
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "bounds"}
        d["bounds"] = list(self.bounds)
        return d


_P = C.c_void_p
_I64P = C.POINTER(C.c_int64)
_IP = C.POINTER(C.c_int)
_DP = C.POINTER(C.c_double)

# name -> (argtypes); every function returns cufsp_status (int) unless listed in _RESTYPE
SIGNATURES = {
    "cufsp_status_string": [C.c_int],
    "cufsp_last_error": [],
    "cufsp_num_states": [C.c_int, _IP, _I64P],
    "cufsp_indx2state": [C.c_int64, _IP, C.c_int, _IP],
    "cufsp_state2indx": [_IP, C.c_int, _IP, _I64P],
    "cufsp_get_states": [C.c_int, _IP, _P, _P],
    "cufsp_mat_create": [C.POINTER(ModelDesc), C.c_int, C.POINTER(_P)],
    "cufsp_mat_destroy": [_P],
    "cufsp_mat_num_states": [_P, _I64P],
    "cufsp_mat_dims": [_P, _IP, _IP, _IP],
    "cufsp_mat_action": [_P, C.c_double, _P, _P, _P],
    "cufsp_mat_apply": [_P, C.c_double, _DP, C.c_double, _P, C.c_double, _P, _P],
    "cufsp_mat_apply_transpose": [_P, C.c_double, _DP, C.c_double, _P, _P, _P],
    "cufsp_mat_action_host": [_P, C.c_double, _P, _P],
    "cufsp_mat_export_propensities": [_P, _P, _P],
    "cufsp_mat_watchdog": [_P, _IP],
    "cufsp_mat_describe": [_P, C.c_char_p, C.c_size_t],
    "cufsp_expv_create": [C.c_int64, C.c_int, C.c_double, C.c_int, C.c_int, C.c_double, C.POINTER(_P)],
    "cufsp_expv_destroy": [_P],
    "cufsp_expv_set_limits": [_P, C.c_int64, C.c_int64],
    "cufsp_expv_bind_mat": [_P, _P, C.c_double],
    "cufsp_expv_bind_mat_coefs": [_P, _P, _DP],
    "cufsp_expv_bind_matvec": [_P, MATVEC_FN, _P],
    "cufsp_expv_set_final_time": [_P, C.c_double],
    "cufsp_expv_solve": [_P, _P, _P, C.POINTER(ExpvStats)],
    "cufsp_expv_step": [_P, _P, _P],
    "cufsp_expv_reset_time": [_P],
    "cufsp_expv_final_time_reached": [_P, _IP],
    "cufsp_expv_get_stats": [_P, C.POINTER(ExpvStats)],
    "cufsp_expm_host": [C.c_int, _DP, _DP],
    "cufsp_expm_blocktri_host": [C.c_int, C.c_int, _DP, _DP],
    "cufsp_bdf_create": [_P, _DP, C.c_double, C.c_double, C.c_int, C.POINTER(_P)],
    "cufsp_bdf_destroy": [_P],
    "cufsp_bdf_set_options": [_P, C.c_double, C.c_double, C.c_double, C.c_int64],
    "cufsp_bdf_set_coefs": [_P, _DP],
    "cufsp_bdf_init": [_P, C.c_double, _P, _P],
    "cufsp_bdf_advance": [_P, C.c_double, _P, C.c_int, _P, _DP],
    "cufsp_bdf_get_stats": [_P, C.POINTER(BdfStats)],
    "cufsp_solver_create": [_P, _DP, C.c_int, C.c_double, _DP, C.c_double, C.c_int, C.c_int, C.c_int, C.POINTER(_P)],
    "cufsp_solver_create_bdf": [_P, _DP, C.c_int, C.c_double, _DP, C.c_double, C.c_double, C.POINTER(_P)],
    "cufsp_solver_destroy": [_P],
    "cufsp_solver_set_coefs": [_P, _DP],
    "cufsp_solver_next_time": [_P, _P, _P, C.POINTER(SolverStatus)],
    "cufsp_solver_solve": [_P, _P, _P, C.POINTER(SolverStatus)],
    "cufsp_solver_reset_time": [_P],
    "cufsp_loglik": [C.c_int64, _P, C.c_int64, _P, _DP, _P],
    "cufsp_likelihood_eval": [_P, _DP, C.c_int, _DP, _P, C.c_int64, _P, C.c_int, C.c_double, _DP, _DP, _P],
    "cufsp_mat_create_table": [C.POINTER(ModelDesc), C.c_int, _DP, C.POINTER(_P)],
    "cufsp_likelihood_grad": [_P, _DP, C.c_int, _DP, _P, C.c_int64, _P, C.c_int, C.c_double, _DP, _DP, _P],
    "cufsp_likelihood_grad_batched": [C.POINTER(ModelDesc), C.c_int, _DP, C.c_int, _DP, _P, C.c_int64, _P, C.c_int,
                                      C.c_double, C.c_int, _DP, _DP],
    "cufsp_ssa": [C.POINTER(ModelDesc), _DP, _IP, _DP, C.c_int, C.c_int, C.c_ulonglong, C.c_int64, _P, _P],
    "cufsp_vec_sum": [C.c_int64, _P, _DP, _P],
    "cufsp_vec_copy": [C.c_int64, _P, _P, _P],
    "cufsp_adaptive_create": [C.POINTER(ModelDesc), _IP, C.c_double, C.c_double, _DP, _DP, C.c_int, C.c_double,
                              C.c_int, C.POINTER(_P)],
    "cufsp_adaptive_destroy": [_P],
    "cufsp_adaptive_set_initial": [_P, _P, _P],
    "cufsp_adaptive_next_time": [_P, _P, C.POINTER(AdaptiveStatus)],
    "cufsp_adaptive_solution": [_P, C.POINTER(C.c_void_p), _IP, _I64P],
    "cufsp_batch_create": [C.POINTER(BatchDesc), C.c_int, C.c_double, C.c_int, C.c_int, C.POINTER(_P)],
    "cufsp_batch_destroy": [_P],
    "cufsp_batch_layout": [_P, _I64P],
    "cufsp_batch_set_coefs": [_P, _DP],
    "cufsp_batch_set_limits": [_P, C.c_int, C.c_int],
    "cufsp_batch_set_shape": [_P, C.c_int, C.c_int],
    "cufsp_batch_solve": [_P, C.c_double, _P, _P, C.POINTER(BatchStat)],
    "cufsp_batch_describe": [_P, C.c_char_p, C.c_size_t],
    "cufsp_vec_sum_noalloc": [C.c_int64, _P, _P, _P],
    "cufsp_cache_trim": [C.POINTER(C.c_size_t)],
}
_RESTYPE = {"cufsp_status_string": C.c_char_p, "cufsp_last_error": C.c_char_p}


def bind(lib: C.CDLL) -> C.CDLL:
    for name, args in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = _RESTYPE.get(name, C.c_int)
    return lib


_lib: C.CDLL | None = None


def load(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load (once) the in-tree libcufsp.so; raise if it is missing."""
    global _lib
    if path is not None:
        return bind(C.CDLL(str(path)))
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m cuda_fsp_b200.build`")
        _lib = bind(C.CDLL(str(LIB_PATH)))
    return _lib


def check(lib: C.CDLL, status: int, where: str) -> None:
    if status != 0:
        detail = lib.cufsp_last_error()
        raise CufspError(status, where, detail.decode() if detail else "")
