"""ADMM on the device (csipm_admm, src/admm.jl) against the reference's
known-answer checks and against the ADMM restatement (oracle_admm.py)."""
import os

import numpy as np
import pytest

import oracle as O
import oracle_admm as OA

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden", "known_answers.npz")


@pytest.mark.parametrize("key", ["100", "200", "500", "16x16", "12x18", "16x24", "32x32", "8x8x8", "6x10x12",
                                 "14x8x4", "8x6x4", "16x16x16"])
@pytest.mark.parametrize("rdft", [True, False])
def test_admm_known_answer(cuda, key, rdft):
    """test/admm_example_{1,2,3}D.jl with check=true: lambda = 0, no mask,
    rho = 1, maxt = 1000, tol = 1e-8 -> ||beta_true - z|| <= 1e-6."""
    import csipm
    torch = cuda
    g = np.load(GOLD)
    size = tuple(int(s) for s in key.split("x"))
    params = csipm.FFTParameters(len(size), size, torch.tensor(g["x_" + key], device="cuda"), 0.0, None)
    op = csipm.FFTOperator(params, rdft=rdft)
    z = csipm.CompressedSensingADMM(params, op, rho=1, maxt=1000, tol=1e-8)
    assert op.admm_stats["status"] == 0
    assert np.linalg.norm(g["beta_" + key] - z.cpu().numpy()) <= 1e-6
    op.close()


def _problem(kind, dims, seed):
    import csipm.problems as P
    spec = P.make_spec(kind, dims=dims, seed=seed)
    op0 = O.Operator(spec.size)
    return P.finalize(spec, op0.A, op0.At)


@pytest.mark.parametrize("kind,dims", [("1d", (2048,)), ("1d", (12000,)), ("2d", (64, 64)), ("2d", (40, 60)),
                                       ("3d", (32, 64, 24)), ("3d", (20, 18, 16))])
def test_admm_matches_oracle(cuda, kind, dims):
    """Masked, lambda > 0, rho = 1, tol = 1e-6: the same iterations as the CPU
    restatement (count within 1) and z within 1e-6 relative."""
    import csipm
    torch = cuda
    prob = _problem(kind, dims, seed=7)
    size = prob.size
    params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
    op = csipm.FFTOperator(params)
    z = csipm.CompressedSensingADMM(params, op, rho=1.0, maxt=1000, tol=1e-6).cpu().numpy()
    st = op.admm_stats
    op.close()
    cop = O.Operator(size, prob.spec.keep)
    zc, info = OA.admm(cop, cop.At(prob.z0), prob.lam, rho=1.0, maxt=1000, tol=1e-6)
    assert st["status"] == 0
    assert abs(st["iterations"] - info["iterations"]) <= 1
    assert np.linalg.norm(z - zc) <= 1e-6 * np.linalg.norm(zc)
