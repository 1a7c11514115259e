"""The ADMM restatement (oracle/oracle_admm.py, src/admm.jl) against the
reference's own known-answer checks (test/admm_example_{1,2,3}D.jl with
check=true: no noise, no mask, lambda = 0, rho = 1, maxt = 1000, tol = 1e-8,
||beta_true - z|| <= 1e-6) and a masked, lambda > 0 case against the IPM twin."""
import os

import numpy as np
import pytest

import oracle as O
import oracle_admm as OA
import oracle_ipm as OI

GOLD = os.path.join(os.path.dirname(__file__), "golden", "known_answers.npz")


@pytest.mark.parametrize("key", ["100", "200", "500", "16x16", "12x18", "16x24", "32x32", "8x8x8", "6x10x12",
                                 "14x8x4", "8x6x4", "16x16x16"])
def test_admm_known_answer(key):
    g = np.load(GOLD)
    size = tuple(int(s) for s in key.split("x"))
    op = O.Operator(size)
    z, info = OA.admm(op, op.At(g["x_" + key]), 0.0, rho=1.0, maxt=1000, tol=1e-8)
    assert info["err"] <= 1e-8
    assert np.linalg.norm(g["beta_" + key] - z) <= 1e-6


def test_admm_cg_takes_two_iterations():
    """A'A is an orthogonal projection here, so A'A + rho I has two eigenvalues
    and each x-update CG ends in at most two iterations."""
    rng = np.random.default_rng(3)
    size = (16, 24)
    keep = rng.random(16 * 24) > 0.2
    op = O.Operator(size, keep)
    b = op.At(np.where(keep, rng.standard_normal(16 * 24), 0.0))
    z, info = OA.admm(op, b, 0.1, maxt=20, tol=0.0)
    assert info["cg_iter"] <= 2 * info["iterations"]


def test_admm_matches_ipm_optimum():
    """Masked, lambda > 0: ADMM run to a tight tolerance lands on the LASSO
    optimum the interior-point twin finds."""
    import csipm.problems as P
    spec = P.make_spec("2d", dims=(32, 24), seed=2)
    op0 = O.Operator(spec.size)
    prob = P.finalize(spec, op0.A, op0.At)
    op = O.Operator(spec.size, spec.keep)
    b = op.At(prob.z0)
    z, info = OA.admm(op, b, prob.lam, rho=1.0, maxt=5000, tol=1e-10)
    beta, _, _ = OI.ipm(op, b, prob.lam, float(prob.z0 @ prob.z0), tol=1e-12)
    Fz = OI.lasso_value(op, z, prob.z0, prob.lam)
    Fb = OI.lasso_value(op, beta, prob.z0, prob.lam)
    assert abs(Fz - Fb) <= 1e-8 * abs(Fb)
