"""ORACLE — test infrastructure only (see oracle.py header).

CPU FP64 restatement of the solver layer:

* ``kkt_*``: the MadNLP KKT plugin of src/fft_kkt.jl — condensed operator
  mul! (:27-44), preconditioner mul! (:73-85), full KKT mul! body (:223-246),
  jtprod! (:253-275), build_kkt! (:285-307) and solve_kkt! (:316-350) with a
  preconditioned CG following Krylov.jl 0.10.2's ``cg`` (x0 = 0, M = P, stop
  when sqrt(r'Mr) <= atol + rtol*sqrt(r0'Mr0), itmax = 2n).
* ``ipm``: the primal-dual interior-point method the library runs on the
  device (csipm_solve), step by step: soft-threshold warm start, Mehrotra
  predictor-corrector on the split formulation of src/fft_model.jl:20-34, the
  condensed Newton system of src/fft_kkt.jl with dc eliminated (Schur
  complement A'A + Db, preconditioner 1/(1+Db)), centring sigma =
  min(1, (mu_aff/mu)^3), fraction-to-boundary max(0.99, 1-mu), inexact
  Newton solves with the forcing term min(cg_rtol, max(1e-6, cg_forcing *
  gap of the previous iteration)), stop on the relative LASSO duality gap or
  on the scaled KKT error max(max(|rd|, |rc|)/max(1, |A'z0|_inf),
  s'z/max(1, |F|)).  MadNLP itself is
  external to the reference and absent here, so this is the CPU twin of the
  GPU algorithm, not a restatement of MadNLP; iteration-count parity with
  MadNLP is unpinned.
* ``fista``: an independent convex check of the LASSO optimum.
"""
from __future__ import annotations

import time

import numpy as np


# ---------------------------------------------------------------------------
# KKT plugin (src/fft_kkt.jl)
# ---------------------------------------------------------------------------

def kkt_build(pr_diag, N):
    """build_kkt! — src/fft_kkt.jl:285-307."""
    S1 = pr_diag[2 * N:3 * N]
    S2 = pr_diag[3 * N:4 * N]
    L1 = S1 + S2
    L2 = S1 - S2
    Minv = 1.0 / (1.0 + L1)
    S = 1.0 / (L1 - L2 ** 2 * Minv)
    P12 = -L2 * S * Minv
    P11 = Minv + Minv * L2 * S * L2 * Minv
    return dict(L1=L1, L2=L2, P11=P11, P12=P12, P22=S)


def condensed_mul(op, K, y, x, alpha, beta):
    """mul!(y, K, x, alpha, beta) — src/fft_kkt.jl:27-44."""
    N = op.N
    xb, xz = x[:N], x[N:]
    Mb = op.AtA(xb)
    out = y.copy()
    out[:N] = beta * y[:N] + alpha * (Mb + K["L1"] * xb + K["L2"] * xz)
    out[N:] = beta * y[N:] + alpha * (K["L2"] * xb + K["L1"] * xz)
    return out


def precond_mul(K, y, x, alpha, beta):
    """mul!(y, P, x, alpha, beta) — src/fft_kkt.jl:73-85."""
    N = K["L1"].size
    xb, xz = x[:N], x[N:]
    out = y.copy()
    out[:N] = beta * y[:N] + alpha * (K["P11"] * xb + K["P12"] * xz)
    out[N:] = beta * y[N:] + alpha * (K["P12"] * xb + K["P22"] * xz)
    return out


def kkt_mul(op, y, x, alpha, beta):
    """mul!(y::KKTVector, kkt, x, alpha, beta) body — src/fft_kkt.jl:223-246
    (MadNLP's _kktmul! diagonal terms, line 248, are the caller's)."""
    N = op.N
    xb, xz, xs1, xs2, xy1, xy2 = (x[i * N:(i + 1) * N] for i in range(6))
    Mb = op.AtA(xb)
    out = y.copy()
    out[0:N] = beta * y[0:N] + alpha * (Mb - xy1 + xy2)
    out[N:2 * N] = beta * y[N:2 * N] - alpha * (xy1 + xy2)
    out[2 * N:3 * N] = beta * y[2 * N:3 * N] - alpha * xy1
    out[3 * N:4 * N] = beta * y[3 * N:4 * N] - alpha * xy2
    out[4 * N:5 * N] = beta * y[4 * N:5 * N] + alpha * (-xb - xz - xs1)
    out[5 * N:6 * N] = beta * y[5 * N:6 * N] + alpha * (xb - xz - xs2)
    return out


def jtprod(x, N):
    """jtprod! — src/fft_kkt.jl:253-275 (first 4N entries)."""
    xy1, xy2 = x[:N], x[N:2 * N]
    return np.concatenate([-xy1 + xy2, -xy1 - xy2, -xy1, -xy2])


def krylov_cg(Amul, b, Mmul=None, atol=1e-12, rtol=0.0, itmax=None):
    """Krylov.jl ``cg`` (0.10.2) semantics: x0 = 0, preconditioned residual norm."""
    n = b.size
    itmax = 2 * n if itmax is None else itmax
    x = np.zeros(n)
    r = b.copy()
    z = Mmul(r) if Mmul else r
    p = z.copy()
    gamma = r @ z
    rNorm = np.sqrt(gamma)
    eps = atol + rtol * rNorm
    it = 0
    solved = rNorm <= eps
    while not solved and it < itmax:
        Ap = Amul(p)
        pAp = p @ Ap
        if pAp <= 0:
            break
        alpha = gamma / pAp
        x += alpha * p
        r -= alpha * Ap
        z = Mmul(r) if Mmul else r
        gnext = r @ z
        rNorm = np.sqrt(gnext)
        it += 1
        solved = rNorm <= eps
        if not solved:
            p = z + (gnext / gamma) * p
        gamma = gnext
    return x, it


def kkt_solve(op, K, w, pr_diag, atol=1e-12, rtol=0.0, preconditioner=True, itmax=None):
    """solve_kkt! body — src/fft_kkt.jl:316-350 (after reduce_rhs!, before finish_aug_solve!)."""
    N = op.N
    S1 = pr_diag[2 * N:3 * N]
    S2 = pr_diag[3 * N:4 * N]
    w1, w2, w3, w4, w5, w6 = (w[i * N:(i + 1) * N].copy() for i in range(6))
    bb = w1 - w3 + w4 - S1 * w5 + S2 * w6
    bz = w2 - w3 - w4 - S1 * w5 - S2 * w6
    b = np.concatenate([bb, bz])
    A = lambda v: condensed_mul(op, K, np.zeros(2 * N), v, 1.0, 0.0)
    M = (lambda v: precond_mul(K, np.zeros(2 * N), v, 1.0, 0.0)) if preconditioner else None
    x, it = krylov_cg(A, b, M, atol=atol, rtol=rtol, itmax=itmax)
    w1 = x[:N]
    w2 = x[N:]
    w5 = -(w3 + S1 * (w1 + w2 + w5))
    w6 = -(w4 + S2 * (-w1 + w2 + w6))
    w3 = (w3 + w5) / S1
    w4 = (w4 + w6) / S2
    return np.concatenate([w1, w2, w3, w4, w5, w6]), it


# ---------------------------------------------------------------------------
# Interior-point solve (CPU twin of csipm_solve)
# ---------------------------------------------------------------------------

def schur_pcg(Qmul, Db, rhs, x0, rtol, maxit, preconditioner=True):
    """(Q + Db) x = rhs, preconditioner 1/(1+Db); stop when sqrt(r'Mr) <= rtol*sqrt(r0'Mr0)."""
    Minv = 1.0 / (1.0 + Db) if preconditioner else np.ones_like(Db)
    if x0 is None:
        x = np.zeros_like(rhs)
        r = rhs.copy()
    else:
        x = x0.copy()
        r = rhs - (Qmul(x) + Db * x)
    p = Minv * r
    rz = r @ p
    thresh = rtol * np.sqrt(rz)
    it = 0
    if np.sqrt(rz) <= thresh:
        return x, it
    while it < maxit:
        q = Qmul(p) + Db * p
        pq = p @ q
        a = rz / pq
        x += a * p
        r -= a * q
        rzn = r @ (Minv * r)
        it += 1
        if not (pq > 0) or not np.isfinite(rzn):
            raise FloatingPointError("CG breakdown")
        if np.sqrt(rzn) <= thresh:
            break
        p = Minv * r + (rzn / rz) * p
        rz = rzn
    return x, it


def _direction(s1, s2, z1, z2, lam, sigmu, cor1, cor2, db):
    D1 = z1 / s1
    D2 = z2 / s2
    L1 = D1 + D2
    L2 = D1 - D2
    h1 = (sigmu - s1 * z1 - cor1) / s1
    h2 = (sigmu - s2 * z2 - cor2) / s2
    rc = lam - z1 - z2
    fc = -rc + h1 + h2
    dc = (fc - L2 * db) / L1
    ds1 = dc + db
    ds2 = dc - db
    dz1 = h1 - D1 * ds1
    dz2 = h2 - D2 * ds2
    return dc, ds1, ds2, dz1, dz2


# floor of the forcing term: the Newton solves are never asked for more than
# FP32 products reach (the mixed-precision solve takes the same iterates)
CG_FORCING_FLOOR = 1e-6


def newton_rtol(cg_rtol, cg_forcing, prev_gap):
    """Relative tolerance of an IPM iteration's Newton solves: the option
    cg_rtol, tightened to cg_forcing * (relative duality gap of the previous
    iteration) but not below CG_FORCING_FLOOR (unless cg_rtol itself is);
    cg_forcing = 0 or no previous iteration: cg_rtol.  Fixed loose solves
    stall once the gap is far below the solve's accuracy (2D 1024^2 at rtol
    1e-2: 116 IPM iterations; with the forcing term, 9)."""
    if cg_forcing <= 0 or prev_gap is None:
        return cg_rtol
    return min(cg_rtol, max(CG_FORCING_FLOOR, cg_forcing * prev_gap))


def ipm(op, b, lam, z0sq, tol=1e-8, max_iter=2000, cg_rtol=1e-8, cg_maxit=None, preconditioner=True,
        verbose=False, cg_forcing=100.0, on_iter=None):
    """Returns (beta, c, info) with info = dict(status, ipm_iter, cg_iter, gap, obj, lasso_obj, mu,
    t_newton, t_newton_products): the last two are the seconds spent in the
    Newton solves and in their products (op.t_matvec when the operator keeps
    it).  on_iter(k, gap), when given, is called after each stop test."""
    N = b.size
    t_newton = 0.0
    t_newton_mv = 0.0

    def newton(*a):
        nonlocal t_newton, t_newton_mv
        t0 = time.perf_counter()
        m0 = getattr(op, "t_matvec", 0.0)
        out = schur_pcg(*a)
        t_newton += time.perf_counter() - t0
        t_newton_mv += getattr(op, "t_matvec", 0.0) - m0
        return out

    cg_maxit = 2 * N if cg_maxit is None else cg_maxit
    Q = op.AtA
    beta = np.where(np.abs(b) - lam > 0, np.copysign(np.abs(b) - lam, b), 0.0)
    maxb = np.abs(beta).max()
    binf = np.abs(b).max()
    # dual start: lambda, floored so that lambda = 0 (the reference's known-answer mode) stays interior
    lz = max(lam, 1e-3 * binf, 1e-12)
    Qb = Q(beta)
    g = np.clip(Qb - b, -0.5 * lz, 0.5 * lz)
    z1 = 0.5 * (lz + g)
    z2 = 0.5 * (lz - g)
    mu0 = 0.1 * lz * max(1e-3, maxb)
    c = np.abs(beta) + mu0 / np.minimum(z1, z2)
    # the slacks s1 = c + beta, s2 = c - beta are kept as variables of their
    # own (MadNLP's slack formulation of the inequality constraints) and take
    # the same steps: recomputing them from c and beta cancels catastrophically
    # once a bound is nearly active
    s1 = c + beta
    s2 = c - beta
    tot_cg = 0
    status = "max_iter"
    info = {}
    k = 0
    prev_gap = None
    while True:
        if k > 0:
            Qb = Q(beta)
        c = 0.5 * (s1 + s2)
        rd = Qb - b - z1 + z2
        rc = lam - z1 - z2
        mu = (s1 @ z1 + s2 @ z2) / (2 * N)
        bb = b @ beta
        bQb = beta @ Qb
        usq = z0sq - 2 * bb + bQb
        F = 0.5 * usq + lam * np.abs(beta).sum()
        ginf = np.abs(b - Qb).max()
        th = min(1.0, lam / ginf) if ginf > 0 else 1.0
        D = th * (z0sq - bb) - 0.5 * th * th * usq
        gap = (F - D) / max(abs(F), 1e-300)
        # scaled KKT error (dual infeasibility, complementarity), the criterion that
        # still applies when lambda = 0 makes the LASSO dual bound degenerate
        kkt = max(max(np.abs(rd).max(), np.abs(rc).max()) / max(1.0, binf), (s1 @ z1 + s2 @ z2) / max(1.0, abs(F)))
        info = dict(gap=gap, kkt=kkt, obj=0.5 * bQb - bb + lam * c.sum(), lasso_obj=F, mu=mu,
                    dual_inf=np.abs(rd).max(), ipm_iter=k, cg_iter=tot_cg)
        if verbose:
            print(f"oracle it {k:3d} mu {mu:.3e} gap {gap:.3e} F {F:.12e} cg {tot_cg}")
        if on_iter is not None:
            on_iter(k, gap)
        if not np.isfinite(gap):
            status = "nonfinite"
            break
        if gap <= tol or kkt <= tol:
            status = "ok"
            break
        if k >= max_iter:
            break
        rt = newton_rtol(cg_rtol, cg_forcing, prev_gap)
        prev_gap = gap
        D1 = z1 / s1
        D2 = z2 / s2
        L1 = D1 + D2
        L2 = D1 - D2
        Db = 4 * D1 * D2 / (D1 + D2)

        def rhs_of(sigmu, cor1, cor2):
            h1 = (sigmu - s1 * z1 - cor1) / s1
            h2 = (sigmu - s2 * z2 - cor2) / s2
            fb = -rd + h1 - h2
            fc = -rc + h1 + h2
            return fb - L2 * fc / L1

        def ratios(d):
            dc, ds1, ds2, dz1, dz2 = d
            def mr(v, dv):
                m = dv < 0
                return (-v[m] / dv[m]).min() if m.any() else np.inf
            return min(mr(s1, ds1), mr(s2, ds2)), min(mr(z1, dz1), mr(z2, dz2))

        dba, it = newton(Q, Db, rhs_of(0.0, 0.0, 0.0), None, rt, cg_maxit, preconditioner)
        tot_cg += it
        aff = _direction(s1, s2, z1, z2, lam, 0.0, 0.0, 0.0, dba)
        minp, mind = ratios(aff)
        a = min(1.0, min(minp, mind))
        _, ds1, ds2, dz1, dz2 = aff
        sz = s1 @ z1 + s2 @ z2
        cross = s1 @ dz1 + ds1 @ z1 + s2 @ dz2 + ds2 @ z2
        dd = ds1 @ dz1 + ds2 @ dz2
        mu_aff = (sz + a * cross + a * a * dd) / (2 * N)
        sigma = min(1.0, max(mu_aff, 0.0) / mu) ** 3
        sigmu = sigma * mu
        cor1 = ds1 * dz1
        cor2 = ds2 * dz2
        db, it = newton(Q, Db, rhs_of(sigmu, cor1, cor2), dba, rt, cg_maxit, preconditioner)
        tot_cg += it
        dirn = _direction(s1, s2, z1, z2, lam, sigmu, cor1, cor2, db)
        minp, mind = ratios(dirn)
        eta = max(0.99, 1.0 - mu)
        ap = min(1.0, eta * minp)
        ad = min(1.0, eta * mind)
        a = min(ap, ad)
        _, ds1, ds2, dz1, dz2 = dirn
        beta = beta + a * db
        s1 = s1 + a * ds1
        s2 = s2 + a * ds2
        z1 = z1 + a * dz1
        z2 = z2 + a * dz2
        k += 1
    c = 0.5 * (s1 + s2)
    info["status"] = status
    info["cg_iter"] = tot_cg
    info["ipm_iter"] = k
    info["t_newton"] = t_newton
    info["t_newton_products"] = t_newton_mv
    return beta, c, info


def fista(op, b, lam, iters=3000, x0=None):
    """Independent LASSO check: FISTA with step 1 (||A'A|| <= 1)."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    y = x.copy()
    t = 1.0
    for _ in range(iters):
        g = op.AtA(y) - b
        v = y - g
        xn = np.sign(v) * np.maximum(np.abs(v) - lam, 0.0)
        tn = (1 + np.sqrt(1 + 4 * t * t)) / 2
        y = xn + (t - 1) / tn * (xn - x)
        x = xn
        t = tn
    return x


def lasso_value(op, beta, z0, lam):
    return 0.5 * np.sum((op.A(beta) - z0) ** 2) + lam * np.abs(beta).sum()
