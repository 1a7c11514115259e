"""The oracle operator and IPM against the reference's own checks (CPU)."""
import numpy as np
import pytest

import oracle as O
import oracle_ipm as OI
from conftest import REF_GRID

GOLD = None


def golden():
    global GOLD
    if GOLD is None:
        import os
        GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "known_answers.npz"))
    return GOLD


@pytest.mark.parametrize("size", REF_GRID)
@pytest.mark.parametrize("rdft", [True, False])
def test_orthonormal_empty_mask(size, rdft):
    """test/unit_tests_ipm.jl:21-29: A'A z = z and norms are preserved with no mask."""
    rng = np.random.default_rng(0)
    z = rng.random(int(np.prod(size)))
    op = O.Operator(size, None, rdft)
    assert np.allclose(op.AtA(z), z, rtol=1e-12, atol=1e-12)
    assert np.isclose(np.linalg.norm(op.At(z)), np.linalg.norm(z), rtol=1e-12)
    assert np.isclose(np.linalg.norm(op.A(z)), np.linalg.norm(z), rtol=1e-12)


@pytest.mark.parametrize("size", REF_GRID)
def test_rdft_matches_full(size):
    rng = np.random.default_rng(1)
    N = int(np.prod(size))
    keep = rng.random(N) > 0.2
    x = rng.standard_normal(N)
    a = O.M_perpt_M_perp_vec(x, size, keep, rdft=True)
    b = O.M_perpt_M_perp_vec(x, size, keep, rdft=False)
    assert np.allclose(a, b, rtol=1e-12, atol=1e-12)


def test_golden_known_answers():
    """beta_true = DFT_to_beta(fft(x)/sqrt(N)) of the reference's known-answer signals."""
    g = golden()
    for k in g.files:
        if not k.startswith("x_"):
            continue
        key = k[2:]
        size = tuple(int(s) for s in key.split("x"))
        beta = O.M_perpt_z(g[k], size)
        assert np.allclose(beta, g["beta_" + key], rtol=0, atol=1e-11)


@pytest.mark.parametrize("key", ["100", "200", "16x16", "12x18", "8x8x8", "6x10x12"])
def test_ipm_known_answer(key):
    """test/ipm_example_{1,2,3}D.jl check=true: lambda=0, no mask -> ||beta - beta_true|| <= 1e-6."""
    g = golden()
    size = tuple(int(s) for s in key.split("x"))
    op = O.Operator(size)
    z0 = g["x_" + key]
    b = op.At(z0)
    beta, c, info = OI.ipm(op, b, 0.0, float(z0 @ z0), tol=1e-10)
    assert info["status"] == "ok"
    assert np.linalg.norm(beta - g["beta_" + key]) <= 1e-6


def test_ipm_matches_fista_masked():
    """Independent convex check of the oracle IPM on a masked, noisy 1D problem."""
    from csipm import problems as P
    spec = P.make_spec("1d", dims=(512,), seed=3)
    op0 = O.Operator(spec.size)
    prob = P.finalize(spec, op0.A, op0.At)
    op = O.Operator(spec.size, spec.keep)
    b = op.At(prob.z0)
    beta, c, info = OI.ipm(op, b, prob.lam, float(prob.z0 @ prob.z0), tol=1e-12)
    assert info["status"] == "ok"
    xf = OI.fista(op, b, prob.lam, iters=4000)
    Fi = OI.lasso_value(op, beta, prob.z0, prob.lam)
    Ff = OI.lasso_value(op, xf, prob.z0, prob.lam)
    assert Fi <= Ff * (1 + 1e-10)
    assert abs(Fi - Ff) <= 1e-8 * Fi
    assert abs(info["lasso_obj"] - Fi) <= 1e-9 * Fi


def test_kkt_solve_satisfies_system():
    """solve_kkt! (src/fft_kkt.jl:316-350) returns a direction that zeroes the
    6N KKT residual with the slack diagonals of pr_diag."""
    size = (12, 18)
    N = int(np.prod(size))
    rng = np.random.default_rng(5)
    keep = rng.random(N) > 0.15
    op = O.Operator(size, keep)
    pr = np.ones(4 * N)
    pr[2 * N:] = rng.uniform(0.1, 10.0, 2 * N)
    K = OI.kkt_build(pr, N)
    w = rng.standard_normal(6 * N)
    sol, it = OI.kkt_solve(op, K, w, pr, atol=1e-12, rtol=0.0)
    assert it > 0
    # KKT matrix applied to sol: mul! body plus the slack diagonal (pr_diag on s)
    y = OI.kkt_mul(op, np.zeros(6 * N), sol, 1.0, 0.0)
    y[2 * N:4 * N] += pr[2 * N:4 * N] * sol[2 * N:4 * N]
    assert np.allclose(y, w, rtol=1e-8, atol=1e-8)
