"""ORACLE — test infrastructure only (see oracle.py header).

CPU FP64 restatement of the reference's ADMM solver, src/admm.jl:
``CompressedSensingADMM(fft_parameter, fft_operator; rho, maxt, tol)``
(:8-61) with its x-update ``cg!`` on the operator ``A'A + rho I``
(``MperptMRho``, :1-6) under Krylov.jl 0.10.2's ``cg`` defaults (x0 = 0, no
preconditioner, atol = rtol = sqrt(eps), stop when ||r|| <= atol + rtol*||b||,
itmax = 2n), the soft threshold of :63-76, the dual update and the stopping
rule err = max(||x1 - x0||, ||y1 - y0||, ||z1 - z0||) <= tol (2-norms).
"""
from __future__ import annotations

import numpy as np

EPS_SQRT = float(np.sqrt(np.finfo(np.float64).eps))


def cg(apply, b, atol=EPS_SQRT, rtol=EPS_SQRT, itmax=None):
    """Krylov.jl ``cg`` without preconditioner from x0 = 0; returns (x, iterations)."""
    n = b.size
    itmax = 2 * n if not itmax else itmax
    x = np.zeros_like(b)
    r = b.copy()
    p = r.copy()
    rr = r @ r
    thresh = atol + rtol * np.sqrt(rr)
    it = 0
    if np.sqrt(rr) <= thresh:
        return x, it
    while it < itmax:
        q = apply(p)
        pq = p @ q
        a = rr / pq
        x += a * p
        r -= a * q
        rrn = r @ r
        it += 1
        if np.sqrt(rrn) <= thresh:
            break
        p = r + (rrn / rr) * p
        rr = rrn
    return x, it


def soft_threshold(x, thre):
    """softthreshold_scalar of src/admm.jl:63-71, elementwise."""
    return np.where(x > thre, x - thre, np.where(x < -thre, x + thre, 0.0))


def admm(op, b, lam, rho=1.0, maxt=1000, tol=1e-6):
    """src/admm.jl:8-61.  b = A'z0; returns (z, info) with info = dict(iterations, cg_iter, err)."""
    n = b.size
    x0 = np.ones(n)
    ztemp = np.ones(n)
    y0 = np.zeros(n)
    t = 0
    err = 1.0
    cg_total = 0
    apply = lambda v: op.AtA(v) + rho * v
    while t < maxt and err > tol:
        rhs = b + rho * ztemp - y0
        x1, it = cg(apply, rhs)
        cg_total += it
        z1 = soft_threshold(x1 + y0 / rho, lam / rho)
        y1 = y0 + rho * (x1 - z1)
        err = max(np.linalg.norm(x1 - x0), np.linalg.norm(y1 - y0), np.linalg.norm(z1 - ztemp))
        x0, ztemp, y0 = x1, z1, y1
        t += 1
    return ztemp, dict(iterations=t, cg_iter=cg_total, err=err)
