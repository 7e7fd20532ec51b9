"""ctypes binding of libsiegpu.so (the C-ABI declared in include/sie_gpu.h).

The library is the only compute path: if it is missing or no CUDA device is
present, calls raise :class:`SieError` -- there is no CPU fallback.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsiegpu.so")

SIE_OK = 0
SIE_NOALLOC_MAX_EDGES = 131072
SIE_ERR_ARG = 1
SIE_ERR_CUDA = 2
SIE_ERR_STATE = 3
SIE_ERR_NOMEM = 4
SIE_ERR_MESH = 5
SIE_ERR_NOCONV = 6
SIE_ERR_TIMEOUT = 7
SIE_ERR_NONFINITE = 8

SIE_PMCHWT = 1
SIE_ICTF = 3
SIE_FP64 = 0
SIE_MIXED = 1
SIE_PRECOND_NONE = 0
SIE_PRECOND_NEAR = 1

ERR_NAMES = {
    1: "SIE_ERR_ARG", 2: "SIE_ERR_CUDA", 3: "SIE_ERR_STATE", 4: "SIE_ERR_NOMEM",
    5: "SIE_ERR_MESH", 6: "SIE_ERR_NOCONV", 7: "SIE_ERR_TIMEOUT", 8: "SIE_ERR_NONFINITE",
}


class SieError(RuntimeError):
    """A non-zero status of the C-ABI (the reference prints and stops instead)."""

    def __init__(self, code, msg):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class SieConfig(C.Structure):
    _fields_ = [
        ("lambda_", C.c_double),
        ("eps_r1_re", C.c_double), ("eps_r1_im", C.c_double),
        ("eps_r2_re", C.c_double), ("eps_r2_im", C.c_double),
        ("formulation", C.c_int), ("ngp", C.c_int), ("tree_s_opt", C.c_int),
        ("truncation_number", C.c_int), ("normal_convention", C.c_int), ("fix_itbn", C.c_int),
        ("device", C.c_int), ("dense", C.c_int),
    ]


class SieSolverCfg(C.Structure):
    _fields_ = [
        ("restart", C.c_int), ("max_iterations", C.c_int), ("tolerance", C.c_double),
        ("use_initial_guess", C.c_int), ("precision", C.c_int), ("inner_restart", C.c_int),
        ("inner_tolerance", C.c_double), ("time_limit_s", C.c_double),
    ]


class SieStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int), ("inner_iterations", C.c_int), ("matvecs", C.c_int),
        ("converged", C.c_int), ("backward_error_arnoldi", C.c_double),
        ("backward_error_true", C.c_double), ("seconds", C.c_double),
    ]


# every symbol declared in include/sie_gpu.h
EXPORTS = [
    "sie_config_default", "sie_solver_default", "sie_last_error", "sie_version", "sie_init",
    "sie_info", "sie_setup", "sie_matvec", "sie_matvec_device", "sie_rhs_planewave",
    "sie_incidence", "sie_solve", "sie_solve_device", "sie_precondition_left", "sie_farfield",
    "sie_get_edges", "sie_get_tree", "sie_get_blocks", "sie_get_near_entries", "sie_get_rt",
    "sie_num_directions", "sie_get_timings", "sie_set_stream", "sie_launch_count", "sie_free",
    "sie_farfield_device_noalloc", "sie_solve_direct", "sie_matvec_adjoint", "sie_matvec_adjoint_device",
    "sie_grad", "sie_set_inner_operator", "sie_autotune", "sie_quadrature_rule",
    "sie_set_preconditioner", "sie_precondition_right", "sie_set_level_truncation",
    "sie_solve_direct_mixed", "sie_solve_direct_mixed_device", "sie_release_factors", "sie_invalidate_factors",
    "sie_field_interior",
]

_lib = None


def load(path=None):
    """Load libsiegpu.so (raise if it is missing)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise SieError(SIE_ERR_STATE, f"{p} not built: run specklesim_b200.build.build()")
    lib = C.CDLL(p)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lp = C.POINTER(C.c_longlong)
    vp = C.c_void_p
    sig = {
        "sie_config_default": (None, [C.POINTER(SieConfig)]),
        "sie_solver_default": (None, [C.POINTER(SieSolverCfg)]),
        "sie_last_error": (C.c_char_p, []),
        "sie_version": (C.c_char_p, []),
        "sie_init": (C.c_int, [C.POINTER(SieConfig), dp, C.c_int, ip, C.c_int, C.POINTER(vp)]),
        "sie_info": (C.c_int, [vp, ip, ip, ip, lp]),
        "sie_setup": (C.c_int, [vp]),
        "sie_matvec": (C.c_int, [vp, dp, dp, C.c_int, C.c_int]),
        "sie_matvec_device": (C.c_int, [vp, vp, vp, C.c_int, C.c_int, vp]),
        "sie_rhs_planewave": (C.c_int, [vp, dp, dp, C.c_int, dp]),
        "sie_incidence": (C.c_int, [C.c_double, C.c_double, C.c_int, C.c_int, dp, dp]),
        "sie_quadrature_rule": (C.c_int, [C.c_int, dp, dp, dp, C.POINTER(C.c_int)]),
        "sie_solve": (C.c_int, [vp, dp, dp, C.c_int, C.POINTER(SieSolverCfg), C.POINTER(SieStats)]),
        "sie_solve_device": (C.c_int, [vp, vp, vp, C.c_int, C.POINTER(SieSolverCfg), C.POINTER(SieStats)]),
        "sie_precondition_left": (C.c_int, [vp, dp, dp]),
        "sie_set_preconditioner": (C.c_int, [vp, C.c_int]),
        "sie_set_level_truncation": (C.c_int, [vp, ip, C.c_int]),
        "sie_precondition_right": (C.c_int, [vp, dp, dp]),
        "sie_farfield": (C.c_int, [vp, dp, dp, C.c_int, dp, dp, dp]),
        "sie_field_interior": (C.c_int, [vp, dp, dp, C.c_int, C.c_double, C.c_double, dp, dp]),
        "sie_get_edges": (C.c_int, [vp, ip, ip]),
        "sie_get_tree": (C.c_int, [vp, dp, lp]),
        "sie_get_blocks": (C.c_int, [vp, ip, ip, C.c_int, dp]),
        "sie_get_near_entries": (C.c_int, [vp, ip, ip, C.c_int, dp]),
        "sie_get_rt": (C.c_int, [vp, ip, C.c_int, dp]),
        "sie_num_directions": (C.c_int, [vp, ip]),
        "sie_get_timings": (C.c_int, [vp, dp, C.c_int]),
        "sie_set_stream": (C.c_int, [vp, vp]),
        "sie_launch_count": (C.c_ulonglong, []),
        "sie_free": (C.c_int, [vp]),
        "sie_farfield_device_noalloc": (C.c_int, [vp, vp, vp, C.c_int, vp, vp, vp, vp]),
        "sie_solve_direct": (C.c_int, [vp, dp, dp, C.c_int]),
        "sie_solve_direct_mixed": (C.c_int, [vp, dp, dp, C.c_int, C.c_double, C.c_int, C.POINTER(SieStats)]),
        "sie_solve_direct_mixed_device": (C.c_int, [vp, vp, vp, C.c_int, C.c_double, C.c_int,
                                                    C.POINTER(SieStats), vp]),
        "sie_release_factors": (C.c_int, [vp]),
        "sie_invalidate_factors": (C.c_int, [vp]),
        "sie_matvec_adjoint": (C.c_int, [vp, dp, dp, C.c_int]),
        "sie_set_inner_operator": (C.c_int, [vp, vp]),
        "sie_autotune": (C.c_int, [vp, C.c_int, dp, ip]),
        "sie_matvec_adjoint_device": (C.c_int, [vp, vp, vp, C.c_int, vp]),
        "sie_grad": (C.c_int, [vp, dp, dp, dp, dp, C.c_int, C.POINTER(SieSolverCfg), dp, dp,
                               C.POINTER(SieStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def check(code):
    if code != SIE_OK:
        raise SieError(code, load().sie_last_error().decode())


def dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def iptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def lptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_longlong))


def as_c128(a):
    return np.ascontiguousarray(a, dtype=np.complex128)
