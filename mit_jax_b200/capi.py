"""ctypes bindings of libcg2d.so (declarations: include/cg2d.h).

The library is built in-tree (mit_jax_b200/_build.py) and loaded from this package directory; there is no CPU
fallback: `lib()` raises if the shared object is missing.
"""

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libcg2d.so"

CG2D_OK = 0
CG2D_NOT_CONVERGED = 1
CG2D_NAN = 2
CG2D_BARRIER_TIMEOUT = 3
CG2D_BAD_ARG = 4
CG2D_CUDA_ERROR = 5
CG2D_WORKSPACE_TOO_SMALL = 6
CG2D_UNSUPPORTED = 7
CG2D_INTERNAL_ERROR = 8
NOALLOC_SCRATCH_BYTES = 32 << 20   # CG2D_NOALLOC_SCRATCH_BYTES

PREC_F64 = 0
PREC_MIXED = 1
SUM_ROWBLOCK = 0
SUM_FORTRAN = 1

STATUS_NAMES = {0: "ok", 1: "not_converged", 2: "nan", 3: "barrier_timeout", 4: "bad_arg", 5: "cuda_error",
                6: "workspace_too_small", 7: "unsupported", 8: "internal_error"}

EXPORTED = ("cg2d_topology_create", "cg2d_topology_destroy", "cg2d_default_params", "cg2d_workspace_size",
            "cg2d_solve_groups", "cg2d_solve_f64", "cg2d_workspace_status", "cg2d_apply_operator",
            "cg2d_edge_products", "cg2d_exchange_scalar", "cg2d_status_string", "cg2d_workspace_profile",
            "cg2d_solve_f64_noalloc", "cg2d_adjoint_exact", "cg2d_adjoint_exact_workspace_size",
            "cg2d_update_operator", "cg2d_pressure_rhs", "cg2d_pressure_post", "cg2d_solve_mixed",
            "cg2d_adjoint_ecco_workspace_size", "cg2d_adjoint_ecco", "cg2d_solve_exact_workspace_size",
            "cg2d_solve_exact", "cg2d_ini_norm")


class Params(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("sum_order", ctypes.c_int), ("rows_per_block", ctypes.c_int),
                ("replace_every", ctypes.c_int), ("replace_above", ctypes.c_double), ("grid_ctas", ctypes.c_int),
                ("ctas_per_sm", ctypes.c_int), ("timeout_s", ctypes.c_double),
                ("test_missing_arrivals", ctypes.c_int), ("profile", ctypes.c_int), ("unit_deal", ctypes.c_int),
                ("stages", ctypes.c_int)]


class Diag(ctypes.Structure):
    _fields_ = [("firstResidual", ctypes.c_double), ("lastResidual", ctypes.c_double), ("sumRHS", ctypes.c_double),
                ("rhsMax", ctypes.c_double), ("numIters", ctypes.c_int32), ("status", ctypes.c_int32),
                ("replacements", ctypes.c_int32), ("reserved", ctypes.c_int32)]


DIAG_BYTES = ctypes.sizeof(Diag)   # 48


class FreeSurf(ctypes.Structure):
    """cg2d_freesurf_t: the FreeSurfParams fields of update_cg2d / cg2d_rhs."""
    _fields_ = [("deltaTMom", ctypes.c_double), ("deltaTFreeSurf", ctypes.c_double),
                ("freeSurfFac", ctypes.c_double), ("implicSurfPress", ctypes.c_double),
                ("implicDiv2DFlow", ctypes.c_double), ("mass2rUnit", ctypes.c_double),
                ("useRealFreshWaterFlux", ctypes.c_int), ("Nr", ctypes.c_int)]

_P = ctypes.c_void_p
_D2 = ctypes.c_void_p * 2


class Group(ctypes.Structure):
    _fields_ = [("topo", _P), ("count", ctypes.c_int), ("nrhs", ctypes.c_int),
                ("aW2d", _P), ("aS2d", _P), ("aC2d", _P), ("pW", _P), ("pS", _P), ("pC", _P),
                ("cg2dNorm", ctypes.c_double), ("cg2dNorm_per_instance", _P),
                ("b", _D2), ("x0", _D2), ("x_out", _D2), ("x_fortran", _D2), ("diag", _D2),
                ("tolerance", ctypes.c_double * 2), ("max_iters", ctypes.c_int * 2)]


_LIB = None


def lib():
    """The loaded libcg2d.so (raises when it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m mit_jax_b200._build` "
                           "(there is no CPU fallback)")
    L = ctypes.CDLL(os.fspath(LIB_PATH))
    i, d = ctypes.c_int, ctypes.c_double
    L.cg2d_topology_create.argtypes = [i, i, i, i, i, _P, _P, ctypes.POINTER(_P)]
    L.cg2d_topology_create.restype = i
    L.cg2d_topology_destroy.argtypes = [_P]
    L.cg2d_topology_destroy.restype = i
    L.cg2d_default_params.argtypes = [ctypes.POINTER(Params)]
    L.cg2d_default_params.restype = None
    L.cg2d_workspace_size.argtypes = [ctypes.POINTER(Group), i, ctypes.POINTER(Params)]
    L.cg2d_workspace_size.restype = ctypes.c_size_t
    L.cg2d_solve_groups.argtypes = [ctypes.POINTER(Group), i, ctypes.POINTER(Params), _P, ctypes.c_size_t, _P]
    L.cg2d_solve_groups.restype = i
    L.cg2d_solve_f64.argtypes = [_P, i, d, _P, _P, _P, _P, _P, _P, _P, _P, d, i, _P, _P, _P,
                                 ctypes.POINTER(Params), _P, ctypes.c_size_t, _P]
    L.cg2d_solve_f64.restype = i
    L.cg2d_solve_f64_noalloc.argtypes = [_P, i, d, _P, _P, _P, _P, _P, _P, _P, _P, d, i, _P, _P, _P,
                                         ctypes.POINTER(Params), _P]
    L.cg2d_solve_f64_noalloc.restype = i
    L.cg2d_adjoint_exact_workspace_size.argtypes = [_P, i, i, i]
    L.cg2d_adjoint_exact_workspace_size.restype = ctypes.c_size_t
    L.cg2d_adjoint_exact.argtypes = [_P, i, d, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, i, i, i,
                                     _P, _P, _P, _P, _P, _P, _P, _P, _P, ctypes.c_size_t, _P]
    L.cg2d_adjoint_exact.restype = i
    L.cg2d_workspace_status.argtypes = [_P, _P]
    L.cg2d_workspace_status.restype = i
    L.cg2d_apply_operator.argtypes = [_P, i, d, _P, _P, _P, _P, _P, _P]
    L.cg2d_apply_operator.restype = i
    L.cg2d_edge_products.argtypes = [_P, i, d, _P, _P, _P, _P, _P, _P, _P]
    L.cg2d_edge_products.restype = i
    L.cg2d_exchange_scalar.argtypes = [_P, i, _P, _P, _P]
    L.cg2d_exchange_scalar.restype = i
    L.cg2d_workspace_profile.argtypes = [_P, ctypes.POINTER(Group), i, ctypes.POINTER(Params), _P, i, _P]
    L.cg2d_workspace_profile.restype = i
    L.cg2d_solve_mixed.argtypes = L.cg2d_solve_f64.argtypes
    L.cg2d_solve_mixed.restype = i
    L.cg2d_adjoint_ecco_workspace_size.argtypes = [_P, i, i, ctypes.POINTER(Params)]
    L.cg2d_adjoint_ecco_workspace_size.restype = ctypes.c_size_t
    L.cg2d_adjoint_ecco.argtypes = [_P, i, d, _P] + [_P] * 8 + [d, i, i] + [_P] * 5 + [ctypes.POINTER(Params), _P,
                                                                                     ctypes.c_size_t, _P]
    L.cg2d_adjoint_ecco.restype = i
    L.cg2d_solve_exact_workspace_size.argtypes = [_P, i, i, i, i]
    L.cg2d_solve_exact_workspace_size.restype = ctypes.c_size_t
    L.cg2d_solve_exact.argtypes = [_P, i, d, _P] + [_P] * 8 + [d, i, _P, i, i] + [_P] * 9 + [_P, ctypes.c_size_t, _P]
    L.cg2d_solve_exact.restype = i
    L.cg2d_update_operator.argtypes = [_P, i, ctypes.POINTER(FreeSurf), d, _P, d] + [_P] * 15 + [_P]
    L.cg2d_update_operator.restype = i
    L.cg2d_pressure_rhs.argtypes = [_P, i, ctypes.POINTER(FreeSurf)] + [_P] * 15 + [_P]
    L.cg2d_pressure_rhs.restype = i
    L.cg2d_pressure_post.argtypes = [_P, i, _P, _P, _P, _P, _P]
    L.cg2d_pressure_post.restype = i
    L.cg2d_ini_norm.argtypes = [_P, i, i, d, d] + [_P] * 8 + [_P]
    L.cg2d_ini_norm.restype = i
    L.cg2d_status_string.argtypes = [i]
    L.cg2d_status_string.restype = ctypes.c_char_p
    _LIB = L
    return L


class Cg2dError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        msg = lib().cg2d_status_string(status).decode() if _LIB is not None else str(status)
        super().__init__(f"{what}: {msg} (status {status})" if what else msg)


def check(status, what=""):
    if status != CG2D_OK:
        raise Cg2dError(status, what)


def default_params():
    p = Params()
    lib().cg2d_default_params(ctypes.byref(p))
    return p
