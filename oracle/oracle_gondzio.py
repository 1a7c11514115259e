"""ORACLE — test infrastructure only (see oracle.py header).

CPU FP64 restatement of the Gondzio formulation of the reference,
src/gondzio_model.jl and src/gondzio_kkt.jl: beta = p - q with p, q >= 0 and a
residual variable r (x = [p; q; r], 3N), objective 1/2 r'r + lambda sum(p, q)
(:67-78), gradient [lambda; r] (:80-93), constraint z0 - A(p - q) - r = 0
(:95-110), and the MadNLP KKT plugin: the condensed operator
[A'A + Dp, -A'A; -A'A, A'A + Dq] (gondzio_kkt.jl:28-53), its block
preconditioner (:63-93), the 4N KKT mul! body (:213-248, before MadNLP's
_kktmul!), jtprod! (:250-268), build_kkt! (:278-301) and solve_kkt! (:303-362)
with a preconditioned CG following Krylov.jl 0.10.2 (x0 = 0, M = P, stop when
sqrt(r'Mr) <= atol + rtol*sqrt(r0'Mr0), atol = 1e-12, rtol = 0).
"""
from __future__ import annotations

import numpy as np


def obj(x, n, lam):
    r = x[2 * n:3 * n]
    return 0.5 * float(r @ r) + lam * float(np.sum(x[:2 * n]))


def grad(x, n, lam):
    g = np.empty(3 * n)
    g[:2 * n] = lam
    g[2 * n:] = x[2 * n:3 * n]
    return g


def cons(op, z0, x, n):
    return z0 - op.A(x[:n] - x[n:2 * n]) - x[2 * n:3 * n]


def build(pr_diag, n):
    """Returns (Dp, Dq, P11, P12, P22) (gondzio_kkt.jl:278-301)."""
    reg_p = pr_diag[:n]
    reg_q = pr_diag[n:2 * n]
    inv_p = 1.0 / (1.0 + reg_p)
    S = 1.0 / (1.0 + reg_q - inv_p)
    P12 = inv_p * S
    P11 = inv_p + inv_p * S * inv_p
    return reg_p.copy(), reg_q.copy(), P11, P12, S


def condensed_mul(op, K, x, n):
    Dp, Dq = K[0], K[1]
    t = op.AtA(x[:n] - x[n:])
    return np.concatenate([Dp * x[:n] + t, Dq * x[n:] - t])


def precond_mul(K, x, n):
    P11, P12, P22 = K[2], K[3], K[4]
    return np.concatenate([P11 * x[:n] + P12 * x[n:], P12 * x[:n] + P22 * x[n:]])


def kkt_mul_body(op, x, n, alpha=1.0, beta=0.0, y=None):
    """MadNLP.mul! of gondzio_kkt.jl:213-248 up to (not including) _kktmul!:
    x, y = [p; q; r; y] (4N)."""
    y = np.zeros(4 * n) if y is None else y.copy()
    xp, xq, xr, xy = x[:n], x[n:2 * n], x[2 * n:3 * n], x[3 * n:4 * n]
    tmp = op.At(xy)
    y[:n] = -alpha * tmp + beta * y[:n]
    y[n:2 * n] = alpha * tmp + beta * y[n:2 * n]
    y[2 * n:3 * n] = alpha * (xr - xy) + beta * y[2 * n:3 * n]
    y[3 * n:] = alpha * (op.A(xq - xp) - xr) + beta * y[3 * n:]
    return y


def jtprod(op, x, n):
    tmp = op.At(x)
    return np.concatenate([-tmp, tmp, -x])


def pcg(apply, prec, b, atol=1e-12, rtol=0.0, itmax=None):
    itmax = 2 * b.size if not itmax else itmax
    x = np.zeros_like(b)
    r = b.copy()
    z = prec(r)
    p = z.copy()
    rz = float(r @ z)
    thresh = atol + rtol * np.sqrt(rz)
    it = 0
    if np.sqrt(rz) <= thresh:
        return x, it
    while it < itmax:
        q = apply(p)
        a = rz / float(p @ q)
        x += a * p
        r -= a * q
        z = prec(r)
        rzn = float(r @ z)
        it += 1
        if np.sqrt(rzn) <= thresh:
            break
        p = z + (rzn / rz) * p
        rz = rzn
    return x, it


def kkt_solve(op, K, w, n, preconditioner=True):
    """solve_kkt! after MadNLP.reduce_rhs!: w = [p; q; r; y] (4N); returns (w', iterations)."""
    w = w.copy()
    wp, wq, wr, wy = w[:n], w[n:2 * n], w[2 * n:3 * n], w[3 * n:]
    tmp = op.At(wr + wy)
    rhs = np.concatenate([wp - tmp, wq + tmp])
    prec = (lambda v: precond_mul(K, v, n)) if preconditioner else (lambda v: v)
    x, it = pcg(lambda v: condensed_mul(op, K, v, n), prec, rhs)
    w_r_old = wr.copy()
    dx = x[:n] - x[n:]
    w[:2 * n] = x
    w[2 * n:3 * n] = -wy - op.A(dx)
    w[3 * n:] = w[2 * n:3 * n] - w_r_old
    return w, it
