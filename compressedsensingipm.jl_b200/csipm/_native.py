"""ctypes binding of libcsipm.so (include/csipm.h).

The shared library is built in-tree next to this file.  There is no fallback:
when the library is missing or cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcsipm.so")

CSIPM_OK = 0
CSIPM_ERR_INVALID = -1
CSIPM_ERR_ODD_DIM = -2
CSIPM_ERR_UNSUPPORTED = -3
CSIPM_ERR_OOM = -4
CSIPM_ERR_CUDA = -5
CSIPM_ERR_CG_MAXITER = -6
CSIPM_ERR_NONFINITE = -7
CSIPM_ERR_IPM_MAXITER = -8
CSIPM_ERR_NO_DEVICE = -9

STATUS_NAMES = {
    0: "OK", -1: "INVALID", -2: "ODD_DIM", -3: "UNSUPPORTED", -4: "OOM", -5: "CUDA",
    -6: "CG_MAXITER", -7: "NONFINITE", -8: "IPM_MAXITER", -9: "NO_DEVICE",
}

# every symbol include/csipm.h declares
EXPORTS = (
    "csipm_default_options", "csipm_create", "csipm_destroy", "csipm_last_error", "csipm_get_info",
    "csipm_get_Atz0", "csipm_beta_to_dft", "csipm_dft_to_beta", "csipm_apply_A", "csipm_apply_At",
    "csipm_apply_AtA", "csipm_obj", "csipm_grad", "csipm_cons", "csipm_hprod", "csipm_kkt_build",
    "csipm_condensed_mul", "csipm_precond_mul", "csipm_kkt_mul", "csipm_jtprod", "csipm_kkt_solve",
    "csipm_solve", "csipm_get_timers", "csipm_profile_passes", "csipm_apply_AtA_static", "csipm_trim_pool",
    "csipm_admm", "csipm_gondzio_obj", "csipm_gondzio_grad", "csipm_gondzio_cons", "csipm_gondzio_kkt_build",
    "csipm_gondzio_condensed_mul", "csipm_gondzio_precond_mul", "csipm_gondzio_kkt_mul", "csipm_gondzio_jtprod",
    "csipm_gondzio_kkt_solve", "csipm_footprint", "csipm_server_create", "csipm_server_submit", "csipm_server_poll", "csipm_server_destroy",
    "csipm_solve_batch",
)


class Problem(ctypes.Structure):
    _fields_ = [
        ("dim", ctypes.c_int),
        ("size", ctypes.c_int * 3),
        ("lam", ctypes.c_double),
        ("z0", ctypes.c_void_p),
        ("host_missing", ctypes.POINTER(ctypes.c_int64)),
        ("n_missing", ctypes.c_int64),
    ]


class Options(ctypes.Structure):
    _fields_ = [
        ("rdft", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("preconditioner", ctypes.c_int),
        ("tol", ctypes.c_double),
        ("max_iter", ctypes.c_int),
        ("cg_atol", ctypes.c_double),
        ("cg_rtol", ctypes.c_double),
        ("cg_maxit", ctypes.c_int),
        ("ipm_cg_rtol", ctypes.c_double),
        ("ir_max", ctypes.c_int),
        ("verbose", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("layout", ctypes.c_int),
        ("cuda_graphs", ctypes.c_int),
        ("autotune", ctypes.c_int),
        ("ipm_cg_forcing", ctypes.c_double),
    ]


class Stats(ctypes.Structure):
    _fields_ = [
        ("status", ctypes.c_int),
        ("ipm_iter", ctypes.c_int),
        ("cg_iter", ctypes.c_int),
        ("matvecs", ctypes.c_int),
        ("refinements", ctypes.c_int),
        ("gap", ctypes.c_double),
        ("obj", ctypes.c_double),
        ("lasso_obj", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("dual_inf", ctypes.c_double),
        ("solve_ms", ctypes.c_double),
        ("launches", ctypes.c_longlong),
        ("fallbacks", ctypes.c_int),
        ("resid_pass_ms", ctypes.c_double),
        ("resid_pass_bytes", ctypes.c_double),
        ("resid_pass_launches", ctypes.c_int),
        ("graph_iters", ctypes.c_int),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class AdmmStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("iterations", ctypes.c_int), ("cg_iter", ctypes.c_int),
                ("err", ctypes.c_double), ("solve_ms", ctypes.c_double)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class ServerOptions(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("hbm_budget", ctypes.c_size_t), ("device", ctypes.c_int),
                ("cuda_graphs", ctypes.c_int), ("batch", ctypes.c_int), ("batch_max_n", ctypes.c_longlong)]


class Request(ctypes.Structure):
    _fields_ = [("problem", Problem), ("options", Options), ("beta_out", ctypes.c_void_p), ("tag", ctypes.c_uint64)]


class Result(ctypes.Structure):
    _fields_ = [("tag", ctypes.c_uint64), ("status", ctypes.c_int), ("stats", Stats), ("queue_ms", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("footprint", ctypes.c_size_t), ("message", ctypes.c_char * 160),
                ("group", ctypes.c_int)]



_lib = None


def load(path: str | None = None):
    """Load libcsipm.so and declare every prototype.  Raises if it is missing."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libcsipm.so not built ({p}); run __graft_entry__.build() or make -C csrc")
    L = ctypes.CDLL(p)
    H = ctypes.c_void_p
    D = ctypes.c_void_p          # device pointer
    I = ctypes.c_int
    dbl = ctypes.c_double
    sig = {
        "csipm_default_options": (I, [ctypes.POINTER(Options)]),
        "csipm_create": (I, [ctypes.POINTER(Problem), ctypes.POINTER(Options), ctypes.POINTER(H)]),
        "csipm_destroy": (I, [H]),
        "csipm_last_error": (ctypes.c_char_p, [H]),
        "csipm_get_info": (I, [H, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_size_t)]),
        "csipm_get_Atz0": (I, [H, D]),
        "csipm_beta_to_dft": (I, [I, ctypes.POINTER(I), I, D, D, ctypes.c_void_p]),
        "csipm_dft_to_beta": (I, [I, ctypes.POINTER(I), I, D, D, ctypes.c_void_p]),
        "csipm_apply_A": (I, [H, D, D]),
        "csipm_apply_At": (I, [H, D, D]),
        "csipm_apply_AtA": (I, [H, D, D]),
        "csipm_obj": (I, [H, D, ctypes.POINTER(dbl)]),
        "csipm_grad": (I, [H, D, D]),
        "csipm_cons": (I, [H, D, D]),
        "csipm_hprod": (I, [H, D, D, dbl]),
        "csipm_kkt_build": (I, [H, D]),
        "csipm_condensed_mul": (I, [H, D, D, dbl, dbl]),
        "csipm_precond_mul": (I, [H, D, D, dbl, dbl]),
        "csipm_kkt_mul": (I, [H, D, D, dbl, dbl]),
        "csipm_jtprod": (I, [H, D, D]),
        "csipm_kkt_solve": (I, [H, D, D, ctypes.POINTER(I)]),
        "csipm_solve": (I, [H, D, D, ctypes.POINTER(Stats)]),
        "csipm_solve_batch": (I, [ctypes.POINTER(H), I, ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Stats)]),
        "csipm_get_timers": (I, [H, ctypes.POINTER(dbl), ctypes.POINTER(dbl), ctypes.POINTER(dbl), I]),
        "csipm_profile_passes": (I, [H, D, I, ctypes.POINTER(dbl), ctypes.POINTER(dbl), ctypes.c_char_p, ctypes.POINTER(I)]),
        "csipm_apply_AtA_static": (I, [I, ctypes.POINTER(I), D, D, D, ctypes.c_void_p]),
        "csipm_trim_pool": (I, [I]),
        "csipm_gondzio_obj": (I, [H, D, ctypes.POINTER(dbl)]),
        "csipm_gondzio_grad": (I, [H, D, D]),
        "csipm_gondzio_cons": (I, [H, D, D]),
        "csipm_gondzio_kkt_build": (I, [H, D]),
        "csipm_gondzio_condensed_mul": (I, [H, D, D, dbl, dbl]),
        "csipm_gondzio_precond_mul": (I, [H, D, D, dbl, dbl]),
        "csipm_gondzio_kkt_mul": (I, [H, D, D, dbl, dbl]),
        "csipm_gondzio_jtprod": (I, [H, D, D]),
        "csipm_gondzio_kkt_solve": (I, [H, D, ctypes.POINTER(I)]),
        "csipm_admm": (I, [H, dbl, I, dbl, D, ctypes.POINTER(AdmmStats)]),
        "csipm_footprint": (I, [I, ctypes.POINTER(I), I, ctypes.c_int64, ctypes.POINTER(ctypes.c_size_t)]),
        "csipm_server_create": (I, [ctypes.POINTER(ServerOptions), ctypes.POINTER(H)]),
        "csipm_server_submit": (I, [H, ctypes.POINTER(Request)]),
        "csipm_server_poll": (I, [H, ctypes.POINTER(Result), I, ctypes.POINTER(I), I]),
        "csipm_server_destroy": (I, [H]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if path is None:
        _lib = L
    return L


class CsipmError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"csipm {STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def check(status, handle=None):
    if status != CSIPM_OK:
        msg = load().csipm_last_error(handle)
        raise CsipmError(status, msg.decode() if msg else "")
    return status
