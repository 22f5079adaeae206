"""ctypes binding of libschwinger_amg.so (declared in include/schwinger_amg.h).

The library is built in place by amg_schwingermodel_b200/build.py; loading fails loudly
when it is missing -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libschwinger_amg.so"

AMG_OK = 0
AMG_NOT_CONVERGED = 1
AMG_ERR_INVALID = -1
AMG_ERR_CUDA = -2
AMG_ERR_STATE = -3
AMG_ERR_NOMEM = -4
AMG_ERR_DEVICE_WAIT = -5
AMG_ERR_UNSUPPORTED = -6
AMG_PREC_F64 = 0
AMG_PREC_MIXED = 1
AMG_CYCLE_V = 0
AMG_CYCLE_K = 1
AMG_PRECOND_MG = 0
AMG_PRECOND_SAP = 1
AMG_PRECOND_NONE = 2
AMG_LINKS_F32 = 0
AMG_LINKS_BF16 = 1
AMG_LINKS_F16 = 2
AMG_SETUP_INIT = 0
AMG_SETUP_SMOOTH = 1
AMG_SETUP_ORTHO = 2
AMG_SETUP_LINKS = 3
AMG_SETUP_BOOT = 4
AMG_SETUP_MIXED = 5
AMG_SETUP_PHASES = 6


class AmgParams(C.Structure):
    _fields_ = [
        ("cycle", C.c_int), ("nu1", C.c_int), ("nu2", C.c_int), ("nit", C.c_int), ("sap_tv_iters", C.c_int),
        ("sap_gmres_m", C.c_int), ("sap_gmres_restarts", C.c_int), ("sap_gmres_tol", C.c_double),
        ("sap_tol", C.c_double), ("kcycle_m", C.c_int), ("kcycle_restarts", C.c_int), ("kcycle_tol", C.c_double),
        ("coarse_m", C.c_int), ("coarse_restarts", C.c_int), ("coarse_tol", C.c_double), ("outer_m", C.c_int),
        ("outer_restarts", C.c_int), ("outer_tol", C.c_double), ("precision", C.c_int), ("max_rhs", C.c_int),
        ("tv_seed", C.c_ulonglong), ("autotune", C.c_int), ("link_storage", C.c_int),
    ]


class AmgSolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("converged", C.c_int), ("rel_residual", C.c_double)]


class AmgError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


_lib = None

_P = C.c_void_p
_I = C.c_int
_D = C.c_double

SIGNATURES = {
    "amg_status_string": (C.c_char_p, [_I]),
    "amg_last_error": (C.c_char_p, []),
    "amg_version": (_I, []),
    "amg_params_default": (None, [C.POINTER(AmgParams)]),
    "amg_read_parameters": (_I, [C.c_char_p, _P, _I, C.POINTER(_I)]),
    "amg_create": (_I, [C.POINTER(_P), _I, _I, _I, _P, _D, C.POINTER(AmgParams), _I]),
    "amg_destroy": (_I, [_P]),
    "amg_get_params": (_I, [_P, C.POINTER(AmgParams)]),
    "amg_set_mass": (_I, [_P, _D]),
    "amg_level_info": (_I, [_P, _I, _P]),
    "amg_set_gauge": (_I, [_P, _P]),
    "amg_dirac_apply": (_I, [_P, _P, _P, _I, _I]),
    "amg_dirac_apply_dev": (_I, [_P, _P, _P, _I, _I]),
    "amg_dirac_apply_raw": (_I, [_P, _P, _P, _I, _I, _I, _D, _I, _P]),
    "amg_debug_dirac_wait_test": (_I, [_P, _P, _P, _I, _I, _I]),
    "amg_cg_normal": (_I, [_P, _P, _P, _I, _D, _P]),
    "amg_bicgstab": (_I, [_P, _P, _P, _P, _I, _D, _P]),
    "amg_restrict_raw_noalloc": (_I, [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "amg_dirac_apply_host": (_I, [_P, _P, _P, _I, _I, _I, _D, _I]),
    "amg_set_cycle": (_I, [_P, _I]),
    "amg_set_preconditioner": (_I, [_P, _I]),
    "amg_set_initial_test_vectors": (_I, [_P, _I, _P]),
    "amg_setup": (_I, [_P]),
    "amg_get_test_vectors": (_I, [_P, _I, _P]),
    "amg_get_coarse_links": (_I, [_P, _I, _P, _P, _P]),
    "amg_level_apply": (_I, [_P, _I, _P, _P]),
    "amg_restrict": (_I, [_P, _I, _P, _P]),
    "amg_prolong": (_I, [_P, _I, _P, _P]),
    "amg_sap": (_I, [_P, _I, _P, _P, _I]),
    "amg_level_gmres": (_I, [_P, _I, _P, _P, C.POINTER(_I)]),
    "amg_cycle": (_I, [_P, _I, _P, _P]),
    "amg_kcycle_fgmres": (_I, [_P, _I, _P, _P, C.POINTER(_I)]),
    "amg_solve": (_I, [_P, _P, _P, _I, _P]),
    "amg_solve_dev": (_I, [_P, _P, _P, _I, _P]),
    "amg_solve_stream": (_I, [_P, _I, _P, _P, _I, _P]),
    "amg_solve_many": (_I, [_I, _P, _P, _P, _P, _P]),
    "amg_solve_many_dev": (_I, [_I, _P, _P, _P, _P, _P]),
    "amg_restrict0_mixed_dev": (_I, [_P, _P, _P, _I]),
    "amg_prolong0_mixed_dev": (_I, [_P, _P, _P, _I]),
    "amg_residual_history": (_I, [_P, _P, _I, C.POINTER(_I)]),
    "amg_solve_adjoint": (_I, [_P, _P, _P, _I, _P]),
    "amg_solve_adjoint_dev": (_I, [_P, _P, _P, _I, _P]),
    "amg_force": (_I, [_P, _P, _P, _I, _P]),
    "amg_force_dev": (_I, [_P, _P, _P, _I, _P]),
    "amg_last_timings": (_I, [_P, C.POINTER(_D), C.POINTER(_D)]),
    "amg_autotune_info": (_I, [_P, _P]),
    "amg_autotune_info_n": (_I, [_P, _P, _I]),
    "amg_setup_timings": (_I, [_P, _P, _I]),
    "amg_profile": (_I, [_P, _I]),
    "amg_profile_query": (_I, [_P, _I, C.POINTER(_D), C.POINTER(C.c_longlong), C.POINTER(_D)]),
    "amg_launch_count": (C.c_longlong, []),
    "amg_get_stream": (_P, [_P]),
    "amg_engine_counters": (_I, [_P, _P, _I]),
}

PROF_SLOTS = {"sap": 0, "engine": 1, "restrict": 2, "prolong": 3, "fine_op": 4, "blas": 5, "outer_op": 6}


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} is not built; run `python -m amg_schwingermodel_b200.build`")
        L = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> int:
    if status < 0:
        msg = lib().amg_last_error().decode(errors="replace")
        raise AmgError(status, where, msg)
    return status


def default_params(**over) -> AmgParams:
    p = AmgParams()
    lib().amg_params_default(C.byref(p))
    for k, v in over.items():
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p
