"""Mixed precision (CSIPM_MIXED): FP32 operator and CG corrections, FP64
residuals, refinement and interior-point logic.  The FP64 device solve of the
same problem is the oracle: beta within 1e-6 relative, objective within 1e-8
relative, iteration count within 2."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _problem(kind, dims, seed):
    import csipm.problems as P
    spec = P.make_spec(kind, dims=dims, seed=seed)
    op0 = O.Operator(spec.size)
    return P.finalize(spec, op0.A, op0.At)


def _solve(torch, prob, precision, **kw):
    import csipm
    size = prob.size
    params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
    nlp = csipm.FFTNLPModel(params, rdft=True, precision=precision, **kw)
    res = csipm.ipm_solve(nlp)
    assert res.status == 0, res.stats
    return res


# solver order (second dimension 64/128/160/256/320) and reference order
# (Stockham FP32 passes), 1D row passes
@pytest.mark.parametrize("kind,dims", [("1d", (4096,)), ("1d", (24000,)), ("2d", (64, 64)), ("2d", (96, 128)), ("3d", (32, 32, 32)),
                                       ("3d", (32, 64, 24)), ("3d", (64, 64, 64)), ("3d", (40, 60, 36))])
@pytest.mark.parametrize("cg_rtol", [1e-8, 1e-5, 1e-2])
def test_mixed_matches_fp64(cuda, kind, dims, cg_rtol):
    """1e-2 runs the loose mode: FP32 Newton directions, corrector warm start
    from the predictor's CG residual, FP64 barrier diagonals only on demand."""
    torch = cuda
    prob = _problem(kind, dims, seed=5)
    r64 = _solve(torch, prob, "fp64", tol=1e-10, ipm_cg_rtol=cg_rtol)
    r32 = _solve(torch, prob, "mixed", tol=1e-10, ipm_cg_rtol=cg_rtol)
    b64, b32 = r64.beta.cpu().numpy(), r32.beta.cpu().numpy()
    assert np.linalg.norm(b32 - b64) / np.linalg.norm(b64) <= 1e-6
    f64, f32 = r64.stats["lasso_obj"], r32.stats["lasso_obj"]
    assert abs(f32 - f64) <= 1e-8 * abs(f64)
    assert abs(r32.stats["ipm_iter"] - r64.stats["ipm_iter"]) <= 2
    if cg_rtol < 1e-6:
        assert r32.stats["refinements"] > 0


def test_mixed_known_answer(cuda):
    """lambda = 0, no mask: the recovered beta is DFT_to_beta(fft(x)/sqrt(N))."""
    import csipm
    torch = cuda
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "known_answers.npz"))
    for key in ("16x16x16", "32x32", "500"):
        size = tuple(int(s) for s in key.split("x"))
        params = csipm.FFTParameters(len(size), size, torch.tensor(g["x_" + key], device="cuda"), 0.0, None)
        nlp = csipm.FFTNLPModel(params, rdft=True, precision="mixed")
        res = csipm.ipm_solve(nlp)
        assert res.status == 0, res.stats
        assert np.linalg.norm(g["beta_" + key] - res.beta.cpu().numpy()) <= 1e-6


def test_mixed_uses_less_fp64_work(cuda):
    """The mixed solve's CG products run in FP32: its FP64 products are the
    per-iteration residuals, warm starts and refinements only."""
    torch = cuda
    prob = _problem("3d", (32, 64, 24), seed=2)
    r32 = _solve(torch, prob, "mixed", tol=1e-10, ipm_cg_rtol=1e-5)
    st = r32.stats
    fp64_products = st["ipm_iter"] + 1 + st["ipm_iter"] + st["refinements"]
    assert st["matvecs"] >= st["cg_iter"]
    assert st["matvecs"] - st["cg_iter"] <= fp64_products


def test_fp32_directions_through_fp64_refinement(cuda):
    """Loose mode with one FP32 CG iteration per round: Newton solves that are
    not done after it leave the FP32 iterate for FP64 refinement rounds and
    come back to FP32 at the end; the solve still matches FP64."""
    torch = cuda
    prob = _problem("3d", (32, 64, 24), seed=3)
    r64 = _solve(torch, prob, "fp64", tol=1e-10, ipm_cg_rtol=1e-2)
    r32 = _solve(torch, prob, "mixed", tol=1e-10, ipm_cg_rtol=1e-2, cg_maxit=1, ir_max=10)
    st = r32.stats
    # FP64 products beyond the per-iteration residual A'A beta: refinement residuals
    assert st["matvecs"] - st["cg_iter"] > st["ipm_iter"] + 1
    b64, b32 = r64.beta.cpu().numpy(), r32.beta.cpu().numpy()
    assert np.linalg.norm(b32 - b64) / np.linalg.norm(b64) <= 1e-6
    assert abs(st["lasso_obj"] - r64.stats["lasso_obj"]) <= 1e-8 * abs(r64.stats["lasso_obj"])
