"""ORACLE — test infrastructure only.

Only tests/, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl
reference`` legs of bench.py import this module, and only as the checker or
as the timed CPU baseline.  The product library never imports it.

CPU FP64 restatement of CompressedSensingIPM.jl's hot path:

* beta <-> DFT maps, three independent statements:
    - ``impl="kern"``  : per-index decode of src/mapping_cpu_kernels.jl (C, maps.c)
    - ``impl="loops"`` : region loops of src/mapping_cpu.jl (C, maps.c)
    - ``impl="wei"``   : slice concatenation of test/fft_wei.jl:21-278 (numpy, below)
* operators A, A^T, A^T A of src/fft_utils.jl:73-123 on FP64 pocketfft
  (scipy.fft), standing in for FFTW 3.3.11 which is not installed;
* model obj/grad/cons of src/fft_model.jl:66-101;
* condensed KKT operator, preconditioner, build_kkt!, solve_kkt! of
  src/fft_kkt.jl:27-85, 213-354 with a preconditioned CG (Krylov.jl 0.10.2
  ``cg`` semantics: stop when sqrt(r'Mr) <= atol + rtol*sqrt(r0'Mr0));
* the primal-dual interior-point loop of this project (oracle_ipm.py).

Arrays follow Julia's column-major layout: a Julia array of size
(N1, N2, N3) is a numpy array of shape (N1, N2, N3) in Fortran order, and flat
vectors are its column-major ravel.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import time

import numpy as np
import scipy.fft as sfft

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liborc_maps.so")
_lib = None

SQRT2 = np.sqrt(2.0)
NCORES = os.cpu_count() or 1


def build():
    """Compile maps.c into _build/liborc_maps.so (gcc, strict IEEE)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        for name in ("orc_loops_dft_to_beta", "orc_kern_dft_to_beta"):
            f = getattr(L, name)
            f.argtypes = [dp, dp, ctypes.c_int, ip, ctypes.c_int]
            f.restype = None
        for name in ("orc_loops_beta_to_dft", "orc_kern_beta_to_dft"):
            f = getattr(L, name)
            f.argtypes = [dp, dp, ctypes.c_int, ip, ctypes.c_int]
            f.restype = None
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _dims(size):
    size = tuple(int(s) for s in size)
    for s in size:
        if s < 2 or s % 2:
            raise ValueError(f"every dimension must be even and >= 2, got {size}")
    return size


def spectrum_shape(size, rdft):
    size = _dims(size)
    if rdft:
        return (size[0] // 2 + 1,) + size[1:]
    return size


# ---------------------------------------------------------------------------
# Maps
# ---------------------------------------------------------------------------

def dft_to_beta(v, size, impl="kern"):
    """DFT_to_beta (src/fft_utils.jl:144-153).  v: complex array (half or full)."""
    size = _dims(size)
    dim = len(size)
    v = np.asarray(v, dtype=np.complex128)
    if impl == "wei":
        return dft_to_beta_wei(v, size)
    vf = np.asfortranarray(v)
    ld1 = vf.shape[0]
    vv = vf.ravel(order="F").view(np.float64).copy()
    beta = np.empty(int(np.prod(size)), dtype=np.float64)
    n = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - dim)))
    f = lib().orc_kern_dft_to_beta if impl == "kern" else lib().orc_loops_dft_to_beta
    f(_dp(beta), _dp(vv), dim, n, ld1)
    return beta


def beta_to_dft(beta, size, rdft=True, impl="kern"):
    """beta_to_DFT (src/fft_utils.jl:195-204).  Returns a Fortran-order complex array."""
    size = _dims(size)
    dim = len(size)
    beta = np.ascontiguousarray(beta, dtype=np.float64)
    if beta.size != int(np.prod(size)):
        raise ValueError("beta has the wrong length")
    if impl == "wei":
        full = beta_to_dft_wei(beta, size)
        return np.asfortranarray(full[: size[0] // 2 + 1]) if rdft else full
    shp = spectrum_shape(size, rdft)
    # cells a map never writes stay NaN so a test sees them
    flat = np.full(2 * int(np.prod(shp)), np.nan, dtype=np.float64)
    n = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - dim)))
    f = lib().orc_kern_beta_to_dft if impl == "kern" else lib().orc_loops_beta_to_dft
    f(_dp(flat), _dp(beta), dim, n, int(bool(rdft)))
    return flat.view(np.complex128).reshape(shp, order="F")


# --- test/fft_wei.jl restatement (numpy slicing on the FULL spectrum) -------

def dft_to_beta_wei(v, size):
    """test/fft_wei.jl:21-132 (reads a full spectrum)."""
    v = np.asarray(v)
    s2 = SQRT2
    if len(size) == 1:
        N = size[0]; M = N // 2
        return np.concatenate([[v[0].real], [v[M].real], s2 * v[1:M].real, s2 * v[1:M].imag])
    if len(size) == 2:
        N1, N2 = size; M1, M2 = N1 // 2, N2 // 2
        F = lambda a: a.reshape(-1, order="F")
        return np.concatenate([
            [v[0, 0].real, v[0, M2].real, v[M1, 0].real, v[M1, M2].real],
            s2 * v[0, 1:M2].real, s2 * v[0, 1:M2].imag,
            s2 * v[M1, 1:M2].real, s2 * v[M1, 1:M2].imag,
            s2 * v[1:M1, 0].real, s2 * v[1:M1, 0].imag,
            s2 * v[1:M1, M2].real, s2 * v[1:M1, M2].imag,
            s2 * F(v[1:M1, 1:M2].real), s2 * F(v[1:M1, 1:M2].imag),
            s2 * F(v[1:M1, M2 + 1:N2].real), s2 * F(v[1:M1, M2 + 1:N2].imag)])
    N1, N2, N3 = size; M1, M2, M3 = N1 // 2, N2 // 2, N3 // 2
    F = lambda a: a.reshape(-1, order="F")
    parts = [np.array([v[0, 0, 0].real, v[0, 0, M3].real, v[0, M2, 0].real, v[0, M2, M3].real,
                       v[M1, 0, 0].real, v[M1, 0, M3].real, v[M1, M2, 0].real, v[M1, M2, M3].real])]
    RI = lambda a: [s2 * F(a.real), s2 * F(a.imag)]
    for (a, b) in ((0, 0), (0, M2), (M1, 0), (M1, M2)):
        parts += RI(v[a, b, 1:M3])
    for (a, c) in ((0, 0), (0, M3), (M1, 0), (M1, M3)):
        parts += RI(v[a, 1:M2, c])
    for (b, c) in ((0, 0), (0, M3), (M2, 0), (M2, M3)):
        parts += RI(v[1:M1, b, c])
    for a in (0, M1):
        parts += RI(v[a, 1:M2, 1:M3]) + RI(v[a, M2 + 1:N2, 1:M3])
    for b in (0, M2):
        parts += RI(v[1:M1, b, 1:M3]) + RI(v[M1 + 1:N1, b, 1:M3])
    for c in (0, M3):
        parts += RI(v[1:M1, 1:M2, c]) + RI(v[M1 + 1:N1, 1:M2, c])
    parts += RI(v[1:M1, 1:M2, 1:M3]) + RI(v[M1 + 1:N1, 1:M2, 1:M3])
    parts += RI(v[1:M1, M2 + 1:N2, 1:M3]) + RI(v[M1 + 1:N1, M2 + 1:N2, 1:M3])
    return np.concatenate(parts)


def _plus(a, b):
    """Julia (a .+ im .* b) ./ sqrt(2), elementwise, with its signed-zero rules."""
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    re = (a + np.copysign(0.0, b)) / SQRT2
    im = b / SQRT2
    return re + 1j * im if re.ndim == 0 else _mk(re, im)


def _minus(a, b):
    """Julia (a .- im .* b) ./ sqrt(2)."""
    a = np.asarray(a, dtype=np.float64); b = np.asarray(b, dtype=np.float64)
    re = (a - np.copysign(0.0, b)) / SQRT2
    im = (-b) / SQRT2
    return _mk(re, im)


def _mk(re, im):
    out = np.empty(np.shape(re), dtype=np.complex128)
    out.real = re
    out.imag = im
    return out


def beta_to_dft_wei(beta, size):
    """test/fft_wei.jl:134-278: builds the FULL spectrum from slices of beta."""
    b = np.asarray(beta, dtype=np.float64)
    cj = np.conj
    if len(size) == 1:
        N = size[0]; M = N // 2
        pos = _plus(b[2:M + 1], b[M + 1:N])
        neg = _minus(b[2:M + 1], b[M + 1:N])[::-1]
        return np.concatenate([[complex(b[0], 0.0)], pos, [complex(b[1], 0.0)], neg])
    if len(size) == 2:
        N1, N2 = size; M1, M2 = N1 // 2, N2 // 2; P1, P2 = M1 - 1, M2 - 1; PP = P1 * P2
        v = np.zeros((N1, N2), dtype=np.complex128, order="F")
        R = lambda a: a.reshape((P1, P2), order="F")
        e = 4 + 4 * P2
        v[:, 0] = np.concatenate([[complex(b[0], 0)], _plus(b[e:e + P1], b[e + P1:e + 2 * P1]),
                                  [complex(b[2], 0)], _minus(b[e:e + P1], b[e + P1:e + 2 * P1])[::-1]])
        o = 4 + 4 * P2 + 4 * P1
        v[:, 1:M2] = np.concatenate([
            _plus(b[4:4 + P2], b[4 + P2:4 + 2 * P2])[None, :],
            R(_plus(b[o:o + PP], b[o + PP:o + 2 * PP])),
            _plus(b[4 + 2 * P2:4 + 3 * P2], b[4 + 3 * P2:4 + 4 * P2])[None, :],
            R(_minus(b[o + 2 * PP:o + 3 * PP], b[o + 3 * PP:o + 4 * PP]))[::-1, ::-1]], axis=0)
        v[:, M2] = np.concatenate([[complex(b[1], 0)], _plus(b[e + 2 * P1:e + 3 * P1], b[e + 3 * P1:e + 4 * P1]),
                                   [complex(b[3], 0)], _minus(b[e + 2 * P1:e + 3 * P1], b[e + 3 * P1:e + 4 * P1])[::-1]])
        v[:, M2 + 1:N2] = np.concatenate([
            cj(v[0, 1:M2])[::-1][None, :],
            cj(v[M1 + 1:N1, 1:M2])[::-1, ::-1],
            cj(v[M1, 1:M2])[::-1][None, :],
            cj(v[1:M1, 1:M2])[::-1, ::-1]], axis=0)
        return v
    # 3D: source slices as in fft_wei.jl:145-278, then the conj mirrors it assigns
    N1, N2, N3 = size; M1, M2, M3 = N1 // 2, N2 // 2, N3 // 2
    P1, P2, P3 = M1 - 1, M2 - 1, M3 - 1
    P23, P13, P12, P123 = P2 * P3, P1 * P3, P1 * P2, P1 * P2 * P3
    v = np.zeros((N1, N2, N3), dtype=np.complex128, order="F")
    cE = 8 + 8 * P3 + 8 * P2                     # i-edges
    cFi = 8 + 8 * P3 + 8 * P2 + 8 * P1           # faces i
    cFj = cFi + 8 * P23                          # faces j
    cFk = cFj + 8 * P13                          # faces k
    cC = cFk + 8 * P12                           # interior
    pr = lambda o, n: _plus(b[o:o + n], b[o + n:o + 2 * n])
    mn = lambda o, n: _minus(b[o:o + n], b[o + n:o + 2 * n])
    R2 = lambda a, s: a.reshape(s, order="F")

    def col_i(vert_lo, vert_hi, off):
        return np.concatenate([[complex(b[vert_lo], 0)], pr(off, P1), [complex(b[vert_hi], 0)], mn(off, P1)[::-1]])

    # lines 151-222 : the (i, j) planes k = 1 and k = M3+1 (full columns in i)
    for (kk, vlo0, vhi0, vlo1, vhi1, eo0, eo1, jo, fo) in (
            (0, 0, 4, 2, 6, cE + 0 * P1, cE + 4 * P1, 8 + 8 * P3 + 0 * P2, cFk + 0 * P12),
            (M3, 1, 5, 3, 7, cE + 2 * P1, cE + 6 * P1, 8 + 8 * P3 + 2 * P2, cFk + 4 * P12)):
        v[:, 0, kk] = col_i(vlo0, vhi0, eo0)
        v[:, 1:M2, kk] = np.concatenate([
            pr(jo, P2)[None, :],
            R2(pr(fo, P12), (P1, P2)),
            pr(jo + 4 * P2, P2)[None, :],
            R2(pr(fo + 2 * P12, P12), (P1, P2))], axis=0)
        v[:, M2, kk] = col_i(vlo1, vhi1, eo1)
        v[:, M2 + 1:N2, kk] = np.concatenate([
            cj(v[0, 1:M2, kk])[::-1][None, :],
            cj(v[M1 + 1:N1, 1:M2, kk])[::-1, ::-1],
            cj(v[M1, 1:M2, kk])[::-1][None, :],
            cj(v[1:M1, 1:M2, kk])[::-1, ::-1]], axis=0)
    # lines 225-262 : the (i, k) planes j = 1 and j = M2+1 for k in 2..M3, and their mirrors
    for (jj, ko, fo) in ((0, 8 + 0 * P3, cFj + 0 * P13), (M2, 8 + 2 * P3, cFj + 4 * P13)):
        v[:, jj, 1:M3] = np.concatenate([
            pr(ko, P3)[None, :],
            R2(pr(fo, P13), (P1, P3)),
            pr(ko + 4 * P3, P3)[None, :],
            R2(pr(fo + 2 * P13, P13), (P1, P3))], axis=0)
        v[:, jj, M3 + 1:N3] = np.concatenate([
            cj(v[0, jj, 1:M3])[::-1][None, :],
            cj(v[M1 + 1:N1, jj, 1:M3])[::-1, ::-1],
            cj(v[M1, jj, 1:M3])[::-1][None, :],
            cj(v[1:M1, jj, 1:M3])[::-1, ::-1]], axis=0)
    # lines 264-272 : planes i = 1 and i = M1+1, interior (j, k)
    for (ii, fo) in ((0, cFi), (M1, cFi + 4 * P23)):
        v[ii, 1:M2, 1:M3] = R2(pr(fo, P23), (P2, P3))
        v[ii, M2 + 1:N2, 1:M3] = R2(pr(fo + 2 * P23, P23), (P2, P3))
        v[ii, 1:M2, M3 + 1:N3] = cj(v[ii, M2 + 1:N2, 1:M3])[::-1, ::-1]
        v[ii, M2 + 1:N2, M3 + 1:N3] = cj(v[ii, 1:M2, 1:M3])[::-1, ::-1]
    # lines 274-284 : interior blocks and their mirrors
    s3 = (P1, P2, P3)
    v[1:M1, 1:M2, 1:M3] = R2(pr(cC, P123), s3)
    v[M1 + 1:N1, M2 + 1:N2, M3 + 1:N3] = cj(v[1:M1, 1:M2, 1:M3])[::-1, ::-1, ::-1]
    v[M1 + 1:N1, 1:M2, 1:M3] = R2(pr(cC + 2 * P123, P123), s3)
    v[1:M1, M2 + 1:N2, M3 + 1:N3] = cj(v[M1 + 1:N1, 1:M2, 1:M3])[::-1, ::-1, ::-1]
    v[1:M1, M2 + 1:N2, 1:M3] = R2(pr(cC + 4 * P123, P123), s3)
    v[M1 + 1:N1, 1:M2, M3 + 1:N3] = cj(v[1:M1, M2 + 1:N2, 1:M3])[::-1, ::-1, ::-1]
    v[M1 + 1:N1, M2 + 1:N2, 1:M3] = R2(pr(cC + 6 * P123, P123), s3)
    v[1:M1, 1:M2, M3 + 1:N3] = cj(v[M1 + 1:N1, M2 + 1:N2, 1:M3])[::-1, ::-1, ::-1]
    return v


# ---------------------------------------------------------------------------
# Operators  (src/fft_utils.jl:73-123), FP64 pocketfft
# ---------------------------------------------------------------------------

def _axes(dim):
    return tuple(range(dim - 1, -1, -1))   # last listed axis (axis 0 = Julia dim 1) is halved by rfftn


def mask_from_missing(size, index_missing):
    """Boolean keep-mask (True = observed) from 0-based linear missing indices."""
    keep = np.ones(int(np.prod(size)), dtype=bool)
    if index_missing is not None and len(index_missing):
        keep[np.asarray(index_missing, dtype=np.int64)] = False
    return keep


def M_perp_beta(beta, size, keep=None, rdft=True, workers=1):
    """A*beta = P_Omega(sqrt(N) * Re(ifft(B beta)))  — src/fft_utils.jl:95-117."""
    size = _dims(size); N = int(np.prod(size)); dim = len(size)
    v = beta_to_dft(beta, size, rdft=rdft)
    if rdft:
        x = sfft.irfftn(v, s=size[::-1], axes=_axes(dim), workers=workers)
    else:
        x = sfft.ifftn(v, axes=_axes(dim), workers=workers).real
    x = (x * np.sqrt(N)).ravel(order="F")
    if keep is not None:
        x = np.where(keep, x, 0.0)
    return x


def M_perpt_z(z, size, rdft=True, workers=1):
    """A^T z = B^T(rfft(z) / sqrt(N)), no mask — src/fft_utils.jl:73-93."""
    size = _dims(size); N = int(np.prod(size)); dim = len(size)
    zz = np.asarray(z, dtype=np.float64).reshape(size, order="F")
    if rdft:
        v = sfft.rfftn(zz, axes=_axes(dim), workers=workers)
    else:
        v = sfft.fftn(zz.astype(np.complex128), axes=_axes(dim), workers=workers)
    v = v / np.sqrt(N)
    return dft_to_beta(v, size)


def M_perpt_M_perp_vec(x, size, keep=None, rdft=True, workers=1):
    """A^T A x — src/fft_utils.jl:67-71, 119-123."""
    return M_perpt_z(M_perp_beta(x, size, keep, rdft, workers), size, rdft, workers)


class Operator:
    """Bundles size / mask / rdft the way FFTOperator does (src/fft_utils.jl:16-54)."""

    def __init__(self, size, keep=None, rdft=True, workers=1):
        self.size = _dims(size)
        self.N = int(np.prod(self.size))
        self.keep = keep
        self.rdft = rdft
        self.workers = workers
        self.n_matvec = 0
        self.t_matvec = 0.0        # seconds spent in AtA (the CPU baseline's unit costs)

    def A(self, beta):
        return M_perp_beta(beta, self.size, self.keep, self.rdft, self.workers)

    def At(self, z):
        return M_perpt_z(z, self.size, self.rdft, self.workers)

    def AtA(self, x):
        self.n_matvec += 1
        t0 = time.perf_counter()
        y = M_perpt_M_perp_vec(x, self.size, self.keep, self.rdft, self.workers)
        self.t_matvec += time.perf_counter() - t0
        return y
