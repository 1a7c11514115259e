"""Parity at the sizes the library is measured on, against the oracle.

* The FP64 operator A, A^T and A^T A at 320^3 with the punched-lattice mask
  and at 2D 1024^2 with the disk lattice plus 5% random missing pixels,
  within 1e-12 relative (2-norm) of pocketfft (src/fft_utils.jl:67-123).
* Full FP64 solves of the 2D 1024^2 workload and of a 128^3 instance of the
  3D generator against the CPU twin (oracle_ipm.ipm) of the same seed: beta
  within 1e-6 relative, objective within 1e-8 relative, IPM iterations within
  1, at the settings the benchmark runs (relative gap 1e-10, inexact Newton
  solves at CG rtol 1e-2).
* Solves and operators whose dimension-2/3 lengths have no two-level factor
  pair (96, 192, 60, 384, 720: the persistent Stockham passes the serving mix
  reaches), FP64 and mixed, against the twin.
* The headline workload, the 320^3 mixed-precision solve, against an FP64 CPU
  twin solve of the same seed (one run: about three minutes of host time).

The oracle runs its FFTs on every host core (pocketfft workers)."""
import os

import numpy as np
import pytest

import oracle as O
import oracle_ipm as OI

pytestmark = pytest.mark.gpu

OP_TOL = 1e-12
CORES = os.cpu_count() or 1


def relerr(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _problem(kind, dims, seed):
    """The measured workloads' generator (csipm.problems), synthesised with the oracle."""
    import csipm.problems as P
    spec = P.make_spec(kind, dims=dims, seed=seed)
    op0 = O.Operator(spec.size, None, True, workers=CORES)
    return P.finalize(spec, op0.A, op0.At)


@pytest.mark.parametrize("kind,dims", [("3d", (320, 320, 320)), ("2d", (1024, 1024)),
                                       ("3d", (60, 96, 192)), ("2d", (720, 384))])
def test_operator_at_measured_sizes(cuda, kind, dims):
    import csipm
    import csipm.problems as P
    torch = cuda
    spec = P.make_spec(kind, dims=dims, seed=5)
    size, keep = spec.size, spec.keep
    N = spec.N
    rng = np.random.default_rng(17)
    z0 = np.where(keep, rng.standard_normal(N), 0.0)
    params = csipm.FFTParameters(len(size), size, torch.tensor(z0, device="cuda"), 0.1, np.flatnonzero(~keep))
    op = csipm.FFTOperator(params, rdft=True)
    ref = O.Operator(size, keep, True, workers=CORES)
    x = rng.standard_normal(N)
    xt = torch.tensor(x, device="cuda")
    assert relerr(op.M_perp_beta(xt).cpu().numpy(), ref.A(x)) <= OP_TOL
    assert relerr(op.M_perpt_z(xt).cpu().numpy(), ref.At(x)) <= OP_TOL
    assert relerr(op.M_perpt_M_perp_vec(xt).cpu().numpy(), ref.AtA(x)) <= OP_TOL
    op.close()


def _gpu_solve(torch, prob, precision, tol, cg_rtol):
    import csipm
    size = prob.size
    params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
    nlp = csipm.FFTNLPModel(params, rdft=True, precision=precision, tol=tol, ipm_cg_rtol=cg_rtol)
    res = csipm.ipm_solve(nlp)
    assert res.status == 0, res.stats
    beta = res.beta.cpu().numpy()
    nlp.op_fft.close()
    return beta, res.stats


def _twin(prob, tol, cg_rtol):
    op = O.Operator(prob.size, prob.spec.keep, True, workers=CORES)
    b = op.At(prob.z0)
    beta, _, info = OI.ipm(op, b, prob.lam, float(prob.z0 @ prob.z0), tol=tol, cg_rtol=cg_rtol)
    assert info["status"] == "ok", info
    return op, beta, info


def _check(op, prob, bg, stats, beta, info, iters):
    assert relerr(bg, beta) <= 1e-6
    Fg = OI.lasso_value(op, bg, prob.z0, prob.lam)
    Fc = OI.lasso_value(op, beta, prob.z0, prob.lam)
    assert abs(Fg - Fc) <= 1e-8 * abs(Fc)
    assert abs(stats["obj"] - info["obj"]) <= 1e-8 * abs(info["obj"])
    assert abs(stats["ipm_iter"] - info["ipm_iter"]) <= iters


@pytest.mark.parametrize("kind,dims", [("2d", (1024, 1024)), ("3d", (128, 128, 128))])
def test_fp64_solve_at_measured_sizes(cuda, kind, dims):
    """The 2D 1024^2 workload and the 3D generator at 128^3: FP64 device solve
    against the CPU twin at the benchmark's settings."""
    torch = cuda
    prob = _problem(kind, dims, seed=0)
    bg, stats = _gpu_solve(torch, prob, "fp64", 1e-10, 1e-2)
    op, beta, info = _twin(prob, 1e-10, 1e-2)
    _check(op, prob, bg, stats, beta, info, iters=1)


@pytest.mark.parametrize("kind,dims", [("3d", (96, 192, 60)), ("2d", (384, 720)), ("3d", (90, 96, 50))])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_off_table_lengths_solve(cuda, kind, dims, precision):
    """Serving-mix sizes whose dimension-2/3 lengths run on the Stockham passes
    (no two-level factor pair), FP64 and mixed, against the twin at the
    serving loop's settings (gap 1e-8 is tightened to 1e-10 here)."""
    torch = cuda
    prob = _problem(kind, dims, seed=2)
    bg, stats = _gpu_solve(torch, prob, precision, 1e-10, 1e-3)
    op, beta, info = _twin(prob, 1e-10, 1e-3)
    _check(op, prob, bg, stats, beta, info, iters=1 if precision == "fp64" else 2)


def test_mixed_320_headline_vs_cpu_twin(cuda):
    """The headline workload: 320^3 punched lattice, seed 0, mixed precision
    (FP32 CG products, FP64 residuals and IPM state) at the benchmark's
    settings, against an FP64 CPU twin solve of the same problem: beta within
    1e-6 relative, objective within 1e-8 relative, IPM iterations within 2."""
    torch = cuda
    prob = _problem("3d", (320, 320, 320), seed=0)
    bg, stats = _gpu_solve(torch, prob, "mixed", 1e-10, 1e-2)
    torch.cuda.empty_cache()
    op, beta, info = _twin(prob, 1e-10, 1e-2)
    _check(op, prob, bg, stats, beta, info, iters=2)
