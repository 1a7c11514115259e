"""csipm — B200-native matrix-free interior-point hot path of CompressedSensingIPM.jl.

This module mirrors the reference's Julia API for the path (same names,
argument meaning and error behaviour), on top of the C ABI in include/csipm.h.
Vectors are CUDA float64 torch tensors (column-major flattening, 0-based
indices); torch provides device memory and the stream, the arithmetic is the
library's own CUDA kernels.

Reference correspondence (paths inside CompressedSensingIPM.jl):

    FFTParameters          src/fft_utils.jl:1-14
    FFTOperator            src/fft_utils.jl:16-54
    M_perp_beta            src/fft_utils.jl:95-117       (A)
    M_perpt_z              src/fft_utils.jl:73-93        (A^T)
    M_perpt_M_perp_vec     src/fft_utils.jl:67-71        (A^T A)
    beta_to_DFT / DFT_to_beta   src/fft_utils.jl:144-222
    FFTNLPModel            src/fft_model.jl              (obj / grad! / cons!)
    FFTKKTSystem           src/fft_kkt.jl                (build_kkt! / mul! / jtprod! / solve_kkt!)
    ipm_solve              src/CompressedSensingIPM.jl:31-36
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _native
from ._native import CsipmError, check

__all__ = [
    "FFTParameters", "FFTOperator", "FFTNLPModel", "FFTKKTSystem", "SolveResult",
    "M_perp_beta", "M_perpt_z", "M_perpt_M_perp_vec", "beta_to_DFT", "DFT_to_beta",
    "ipm_solve", "CsipmError", "lib",
]


def lib():
    return _native.load()


def _torch():
    import torch
    return torch


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _as_dev64(x, name="vector"):
    torch = _torch()
    if isinstance(x, torch.Tensor):
        if not x.is_cuda:
            raise ValueError(f"{name} must be a CUDA tensor")
        if x.dtype != torch.float64:
            raise ValueError(f"{name} must be float64")
        if not x.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
        return x
    return torch.as_tensor(np.ascontiguousarray(x, dtype=np.float64), device="cuda")


def _stream():
    return _torch().cuda.current_stream().cuda_stream


def _check_size(DFTsize):
    size = tuple(int(s) for s in DFTsize)
    if len(size) not in (1, 2, 3):
        raise ValueError("DFTsize must have 1, 2 or 3 entries")
    for s in size:
        if s < 2 or s % 2:
            raise ValueError(f"every dimension must be even and >= 2, got {size}")
    return size


# --------------------------------------------------------------------- maps
def beta_to_DFT(DFTdim, DFTsize, beta, rdft=False):
    """beta_to_DFT(DFTdim, size, beta; rdft) -> complex128 tensor shaped like
    Julia's array (column-major): (N1/2+1, N2, N3) if rdft else (N1, N2, N3).
    Bit-exact with src/mapping_cpu_kernels.jl."""
    torch = _torch()
    size = _check_size(DFTsize)
    beta = _as_dev64(beta, "beta")
    ni = size[0] // 2 + 1 if rdft else size[0]
    rest = int(np.prod(size[1:])) if len(size) > 1 else 1
    v = torch.empty(2 * ni * rest, dtype=torch.float64, device=beta.device)
    n = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - len(size))))
    check(lib().csipm_beta_to_dft(int(DFTdim), n, int(bool(rdft)), _ptr(beta), _ptr(v), ctypes.c_void_p(_stream())))
    shape = (ni,) + size[1:]
    # Julia column-major (ni, N2, N3) == C-order (N3, N2, ni)
    return torch.view_as_complex(v.view(-1, 2)).view(shape[::-1]).permute(*reversed(range(len(shape))))


def DFT_to_beta(DFTdim, DFTsize, v):
    """DFT_to_beta(DFTdim, size, v) -> float64 tensor of length N.  `v` is a
    complex128 tensor in Julia layout (as returned by beta_to_DFT), half or full
    spectrum; only v[0:N1/2+1, ...] is read."""
    torch = _torch()
    size = _check_size(DFTsize)
    if v.dtype != torch.complex128:
        raise ValueError("v must be complex128")
    ld1 = v.shape[0]
    # back to the flat column-major buffer
    flat = v.permute(*reversed(range(v.dim()))).contiguous()
    fr = torch.view_as_real(flat).reshape(-1)
    beta = torch.empty(int(np.prod(size)), dtype=torch.float64, device=v.device)
    n = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - len(size))))
    check(lib().csipm_dft_to_beta(int(DFTdim), n, int(ld1), _ptr(fr), _ptr(beta), ctypes.c_void_p(_stream())))
    return beta


# --------------------------------------------------------------------- params
@dataclasses.dataclass
class FFTParameters:
    """FFTParameters(DFTdim, DFTsize, z0, lambda, index_missing) — src/fft_utils.jl:1-14.

    index_missing: 0-based column-major linear indices of the missing samples
    (Julia's 1-based linear indices minus one), or a boolean keep-mask of length N.
    z0 must be zero at the missing samples, as in the reference.
    """
    DFTdim: int
    DFTsize: tuple
    z0: object
    lam: float
    index_missing: object = None

    def missing_indices(self):
        im = self.index_missing
        if im is None:
            return np.zeros(0, dtype=np.int64)
        a = np.asarray(im)
        if a.dtype == bool:
            return np.flatnonzero(~a).astype(np.int64)
        return np.ascontiguousarray(a, dtype=np.int64).ravel()


def _options(rdft=True, precision="fp64", preconditioner=True, tol=1e-8, max_iter=2000, cg_atol=1e-12,
             cg_rtol=0.0, cg_maxit=0, ipm_cg_rtol=1e-8, ir_max=3, verbose=False, stream=None, layout="solver",
             cuda_graphs=True, autotune=True, ipm_cg_forcing=100.0):
    o = _native.Options()
    check(lib().csipm_default_options(ctypes.byref(o)))
    o.rdft = int(bool(rdft))
    o.precision = {"fp64": 0, "mixed": 1}[precision] if isinstance(precision, str) else int(precision)
    o.preconditioner = int(bool(preconditioner))
    o.tol = float(tol)
    o.max_iter = int(max_iter)
    o.cg_atol = float(cg_atol)
    o.cg_rtol = float(cg_rtol)
    o.cg_maxit = int(cg_maxit)
    o.ipm_cg_rtol = float(ipm_cg_rtol)
    o.ir_max = int(ir_max)
    o.verbose = int(bool(verbose))
    o.stream = ctypes.c_void_p(stream if stream is not None else _stream())
    o.layout = {"solver": 0, "reference": 1}[layout] if isinstance(layout, str) else int(layout)
    o.cuda_graphs = int(bool(cuda_graphs))
    o.autotune = int(bool(autotune))
    o.ipm_cg_forcing = float(ipm_cg_forcing)
    return o


class FFTOperator:
    """FFTOperator{VT}(nβ, DFTdim, DFTsize, index_missing, rdft) — src/fft_utils.jl:16-54.

    Owns one library handle (FFT plans, mask, spectrum buffer, workspaces) bound
    to the torch stream current at construction.
    """

    def __init__(self, parameters: FFTParameters, rdft=True, **opts):
        self.parameters = parameters
        self.DFTdim = int(parameters.DFTdim)
        self.DFTsize = _check_size(parameters.DFTsize)
        if len(self.DFTsize) != self.DFTdim:
            raise ValueError("len(DFTsize) must equal DFTdim")
        self.rdft = bool(rdft)
        self.N = int(np.prod(self.DFTsize))
        self.z0 = _as_dev64(parameters.z0, "z0").reshape(-1)
        if self.z0.numel() != self.N:
            raise ValueError("z0 has the wrong length")
        self._missing = parameters.missing_indices()
        prob = _native.Problem()
        prob.dim = self.DFTdim
        for d in range(3):
            prob.size[d] = self.DFTsize[d] if d < self.DFTdim else 1
        prob.lam = float(parameters.lam)
        prob.z0 = self.z0.data_ptr()
        prob.host_missing = self._missing.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))
        prob.n_missing = int(self._missing.size)
        self.options = _options(rdft=rdft, **opts)
        h = ctypes.c_void_p()
        check(lib().csipm_create(ctypes.byref(prob), ctypes.byref(self.options), ctypes.byref(h)))
        self.handle = h
        self.fft_timer = 0.0
        self.mapping_timer = 0.0

    def close(self):
        if getattr(self, "handle", None):
            lib().csipm_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _new(self, n=None):
        torch = _torch()
        return torch.empty(self.N if n is None else n, dtype=torch.float64, device=self.z0.device)

    def device_bytes(self):
        n = ctypes.c_int64()
        b = ctypes.c_size_t()
        check(lib().csipm_get_info(self.handle, ctypes.byref(n), ctypes.byref(b)), self.handle)
        return int(b.value)

    def M_perp_beta(self, beta, out=None):
        beta = _as_dev64(beta, "beta")
        out = self._new() if out is None else out
        check(lib().csipm_apply_A(self.handle, _ptr(beta), _ptr(out)), self.handle)
        return out

    def M_perpt_z(self, z, out=None):
        z = _as_dev64(z, "z").reshape(-1)
        out = self._new() if out is None else out
        check(lib().csipm_apply_At(self.handle, _ptr(z), _ptr(out)), self.handle)
        return out

    def M_perpt_M_perp_vec(self, x, out=None):
        x = _as_dev64(x, "x")
        out = self._new() if out is None else out
        check(lib().csipm_apply_AtA(self.handle, _ptr(x), _ptr(out)), self.handle)
        return out


def M_perp_beta(op: FFTOperator, beta):
    return op.M_perp_beta(beta)


def M_perpt_z(op: FFTOperator, z):
    return op.M_perpt_z(z)


def M_perpt_M_perp_vec(op: FFTOperator, x):
    return op.M_perpt_M_perp_vec(x)


class FFTNLPModel:
    """FFTNLPModel{VT}(parameters; krylov_solver=:cg, rdft=false, preconditioner=true)
    — src/fft_model.jl.  Variables x = [beta; c] (2N), constraints
    [-beta - c; beta - c] <= 0 (2N)."""

    def __init__(self, parameters: FFTParameters, krylov_solver="cg", rdft=False, preconditioner=True, **opts):
        if krylov_solver != "cg":
            raise ValueError("only krylov_solver='cg' is supported (as in the reference)")
        self.parameters = parameters
        self.op_fft = FFTOperator(parameters, rdft=rdft, preconditioner=preconditioner, **opts)
        self.nbeta = self.op_fft.N
        self.nvar = 2 * self.nbeta
        self.ncon = 2 * self.nbeta
        self.preconditioner = preconditioner
        self.krylov_solver = krylov_solver
        self.counters = {"neval_obj": 0, "neval_grad": 0, "neval_cons": 0, "neval_hprod": 0}

    @property
    def handle(self):
        return self.op_fft.handle

    @property
    def M_perpt_z0(self):
        out = self.op_fft._new()
        check(lib().csipm_get_Atz0(self.handle, _ptr(out)), self.handle)
        return out

    def obj(self, x):
        self.counters["neval_obj"] += 1
        x = _as_dev64(x, "x")
        f = ctypes.c_double()
        check(lib().csipm_obj(self.handle, _ptr(x), ctypes.byref(f)), self.handle)
        return f.value

    def grad(self, x, g):
        """grad!(nlp, x, g) — in place on g (2N)."""
        self.counters["neval_grad"] += 1
        check(lib().csipm_grad(self.handle, _ptr(_as_dev64(x, "x")), _ptr(g)), self.handle)
        return g

    def cons(self, x, c):
        """cons!(nlp, x, c) — in place on c (2N)."""
        self.counters["neval_cons"] += 1
        check(lib().csipm_cons(self.handle, _ptr(_as_dev64(x, "x")), _ptr(c)), self.handle)
        return c

    def hprod(self, x, v, hv, obj_weight=1.0):
        """Hessian-of-Lagrangian product [A'A v_beta; 0] * obj_weight (constraints are linear)."""
        self.counters["neval_hprod"] += 1
        check(lib().csipm_hprod(self.handle, _ptr(_as_dev64(v, "v")), _ptr(hv), float(obj_weight)), self.handle)
        return hv


class FFTKKTSystem:
    """The MadNLP KKT plugin of src/fft_kkt.jl over a FFTNLPModel: build_kkt!,
    condensed and preconditioner mul!, the 6N KKT mul!, jtprod! and solve_kkt!.
    krylov_iterations collects the CG iteration count of every solve."""

    def __init__(self, nlp: FFTNLPModel):
        self.nlp = nlp
        self.krylov_iterations = []
        self.krylov_timer = []

    @property
    def handle(self):
        return self.nlp.handle

    def build_kkt(self, pr_diag):
        check(lib().csipm_kkt_build(self.handle, _ptr(_as_dev64(pr_diag, "pr_diag"))), self.handle)

    def condensed_mul(self, y, x, alpha=1.0, beta=0.0):
        check(lib().csipm_condensed_mul(self.handle, _ptr(y), _ptr(_as_dev64(x, "x")), float(alpha), float(beta)), self.handle)
        return y

    def precond_mul(self, y, x, alpha=1.0, beta=0.0):
        check(lib().csipm_precond_mul(self.handle, _ptr(y), _ptr(_as_dev64(x, "x")), float(alpha), float(beta)), self.handle)
        return y

    def mul(self, y, x, alpha=1.0, beta=0.0):
        check(lib().csipm_kkt_mul(self.handle, _ptr(y), _ptr(_as_dev64(x, "x")), float(alpha), float(beta)), self.handle)
        return y

    def jtprod(self, y, x):
        check(lib().csipm_jtprod(self.handle, _ptr(y), _ptr(_as_dev64(x, "x"))), self.handle)
        return y

    def solve_kkt(self, w, pr_diag):
        it = ctypes.c_int()
        check(lib().csipm_kkt_solve(self.handle, _ptr(w), _ptr(_as_dev64(pr_diag, "pr_diag")), ctypes.byref(it)), self.handle)
        self.krylov_iterations.append(int(it.value))
        return w


class GondzioNLPModel:
    """GondzioNLPModel{VT}(parameters; krylov_solver, rdft, preconditioner) —
    src/gondzio_model.jl:12-65: x = [p; q; r] (3N), beta = p - q, one
    constraint block z0 - A(p - q) - r = 0.  obj/grad!/cons! on the device."""

    def __init__(self, parameters: FFTParameters, krylov_solver="cg", rdft=False, preconditioner=True, **opts):
        if krylov_solver != "cg":
            raise ValueError("only krylov_solver='cg' is available")
        self.parameters = parameters
        self.op_fft = FFTOperator(parameters, rdft=rdft, preconditioner=preconditioner, **opts)
        self.nbeta = self.op_fft.N
        self.nvar = 3 * self.nbeta
        self.ncon = self.nbeta
        self.counters = {"neval_obj": 0, "neval_grad": 0, "neval_cons": 0}

    @property
    def handle(self):
        return self.op_fft.handle

    def obj(self, x):
        self.counters["neval_obj"] += 1
        f = ctypes.c_double()
        check(lib().csipm_gondzio_obj(self.handle, _ptr(_as_dev64(x, "x")), ctypes.byref(f)), self.handle)
        return f.value

    def grad(self, x, g):
        self.counters["neval_grad"] += 1
        check(lib().csipm_gondzio_grad(self.handle, _ptr(_as_dev64(x, "x")), _ptr(g)), self.handle)
        return g

    def cons(self, x, c):
        self.counters["neval_cons"] += 1
        check(lib().csipm_gondzio_cons(self.handle, _ptr(_as_dev64(x, "x")), _ptr(c)), self.handle)
        return c


class GondzioKKTSystem:
    """The MadNLP KKT plugin of src/gondzio_kkt.jl over a GondzioNLPModel:
    build_kkt!, condensed and preconditioner mul!, the 4N KKT mul! body,
    jtprod! and solve_kkt! (after MadNLP.reduce_rhs!)."""

    def __init__(self, nlp: GondzioNLPModel):
        self.nlp = nlp
        self.krylov_iterations = []

    @property
    def handle(self):
        return self.nlp.handle

    def build_kkt(self, pr_diag):
        check(lib().csipm_gondzio_kkt_build(self.handle, _ptr(_as_dev64(pr_diag, "pr_diag"))), self.handle)

    def condensed_mul(self, y, x, alpha=1.0, beta=0.0):
        check(lib().csipm_gondzio_condensed_mul(self.handle, _ptr(y), _ptr(_as_dev64(x, "x")), float(alpha),
                                                float(beta)), self.handle)
        return y

    def precond_mul(self, y, x, alpha=1.0, beta=0.0):
        check(lib().csipm_gondzio_precond_mul(self.handle, _ptr(y), _ptr(_as_dev64(x, "x")), float(alpha),
                                              float(beta)), self.handle)
        return y

    def mul(self, y, x, alpha=1.0, beta=0.0):
        check(lib().csipm_gondzio_kkt_mul(self.handle, _ptr(y), _ptr(_as_dev64(x, "x")), float(alpha), float(beta)),
              self.handle)
        return y

    def jtprod(self, y, x):
        check(lib().csipm_gondzio_jtprod(self.handle, _ptr(y), _ptr(_as_dev64(x, "x"))), self.handle)
        return y

    def solve_kkt(self, w):
        it = ctypes.c_int()
        check(lib().csipm_gondzio_kkt_solve(self.handle, _ptr(w), ctypes.byref(it)), self.handle)
        self.krylov_iterations.append(int(it.value))
        return w


@dataclasses.dataclass
class SolveResult:
    solution: object        # 2N tensor [beta; c]
    status: int
    stats: dict

    @property
    def beta(self):
        n = self.solution.numel() // 2
        return self.solution[:n]


def CompressedSensingADMM(parameters: FFTParameters, fft_operator: "FFTOperator", rho=1.0, maxt=1000, tol=1e-6):
    """CompressedSensingADMM(fft_parameter, fft_operator; rho, maxt, tol) —
    src/admm.jl:8-61, on the device (csipm_admm).  Returns z (torch, N); the
    statistics land in ``fft_operator.admm_stats``."""
    torch = _torch()
    n = int(np.prod(parameters.DFTsize))
    z = torch.empty(n, dtype=torch.float64, device=fft_operator.z0.device)
    st = _native.AdmmStats()
    status = lib().csipm_admm(fft_operator.handle, float(rho), int(maxt), float(tol), _ptr(z), ctypes.byref(st))
    if status not in (0, _native.CSIPM_ERR_IPM_MAXITER):
        check(status, fft_operator.handle)
    fft_operator.admm_stats = st.as_dict()
    return z


def ipm_solve_batch(nlps, raise_on_error=False):
    """Solves several FFTNLPModels together (csipm_solve_batch): every step is
    one kernel launch for all of them.  The models must share the dimension
    count, whether they have missing samples and (1D) whether N1/2 > 2048;
    each keeps its own options.  Returns one SolveResult per model."""
    torch = _torch()
    k = len(nlps)
    hs = (ctypes.c_void_p * k)(*[m.handle for m in nlps])
    sols = [torch.empty(2 * m.nbeta, dtype=torch.float64, device=m.op_fft.z0.device) for m in nlps]
    outs = (ctypes.c_void_p * k)(*[s.data_ptr() for s in sols])
    st = (_native.Stats * k)()
    status = lib().csipm_solve_batch(hs, k, outs, st)
    if status not in (0, _native.CSIPM_ERR_IPM_MAXITER) or (raise_on_error and status != 0):
        check(status)
    return [SolveResult(sols[j], int(st[j].status), st[j].as_dict()) for j in range(k)]


def ipm_solve(nlp: FFTNLPModel, raise_on_error=False):
    """ipm_solve!(solver) — src/CompressedSensingIPM.jl:31-36, on the device."""
    torch = _torch()
    n = nlp.nbeta
    sol = torch.empty(2 * n, dtype=torch.float64, device=nlp.op_fft.z0.device)
    st = _native.Stats()
    status = lib().csipm_solve(nlp.handle, _ptr(sol), ctypes.c_void_p(sol.data_ptr() + 8 * n), ctypes.byref(st))
    if raise_on_error and status != 0:
        check(status, nlp.handle)
    if status not in (0, _native.CSIPM_ERR_IPM_MAXITER, _native.CSIPM_ERR_CG_MAXITER) and not raise_on_error:
        check(status, nlp.handle)
    return SolveResult(sol, int(status), st.as_dict())
