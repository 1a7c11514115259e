"""NLPModels and MadNLP KKT-plugin entry points on the GPU against the oracle
restatement of src/fft_model.jl and src/fft_kkt.jl."""
import numpy as np
import pytest

import oracle as O
import oracle_ipm as OI

pytestmark = pytest.mark.gpu


def setup(size=(12, 18), seed=0):
    import csipm
    import torch
    N = int(np.prod(size))
    rng = np.random.default_rng(seed)
    keep = rng.random(N) > 0.15
    z0 = np.where(keep, rng.standard_normal(N), 0.0)
    params = csipm.FFTParameters(len(size), size, torch.tensor(z0, device="cuda"), 0.7, np.flatnonzero(~keep))
    nlp = csipm.FFTNLPModel(params, rdft=True)
    ref = O.Operator(size, keep)
    return nlp, ref, z0, rng, N


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("size", [(100,), (12, 18), (6, 10, 12)])
def test_obj_grad_cons_hprod(cuda, size):
    torch = cuda
    nlp, ref, z0, rng, N = setup(size)
    b = ref.At(z0)
    assert rel(nlp.M_perpt_z0.cpu().numpy(), b) <= 1e-12
    x = rng.standard_normal(2 * N)
    xt = torch.tensor(x, device="cuda")
    beta, c = x[:N], x[N:]
    f_ref = 0.5 * np.sum(ref.A(beta) ** 2) - beta @ b + 0.7 * c.sum()        # src/fft_model.jl:66-75
    assert abs(nlp.obj(xt) - f_ref) <= 1e-11 * max(1.0, abs(f_ref))
    g = torch.empty(2 * N, dtype=torch.float64, device="cuda")
    nlp.grad(xt, g)
    assert rel(g.cpu().numpy(), np.concatenate([ref.AtA(beta) - b, np.full(N, 0.7)])) <= 1e-12
    cc = torch.empty(2 * N, dtype=torch.float64, device="cuda")
    nlp.cons(xt, cc)
    assert np.array_equal(cc.cpu().numpy(), np.concatenate([-beta - c, beta - c]))
    hv = torch.empty(2 * N, dtype=torch.float64, device="cuda")
    nlp.hprod(xt, xt, hv, 2.0)
    assert rel(hv.cpu().numpy(), np.concatenate([2.0 * ref.AtA(beta), np.zeros(N)])) <= 1e-12


def test_kkt_plugin_products(cuda):
    import csipm
    torch = cuda
    nlp, ref, z0, rng, N = setup()
    kkt = csipm.FFTKKTSystem(nlp)
    pr = np.ones(4 * N)
    pr[2 * N:] = rng.uniform(0.05, 20.0, 2 * N)
    prt = torch.tensor(pr, device="cuda")
    kkt.build_kkt(prt)
    K = OI.kkt_build(pr, N)
    x2 = rng.standard_normal(2 * N)
    y2 = rng.standard_normal(2 * N)
    yt = torch.tensor(y2, device="cuda")
    kkt.condensed_mul(yt, torch.tensor(x2, device="cuda"), 1.5, -0.5)
    assert rel(yt.cpu().numpy(), OI.condensed_mul(ref, K, y2, x2, 1.5, -0.5)) <= 1e-12
    yt = torch.tensor(y2, device="cuda")
    kkt.precond_mul(yt, torch.tensor(x2, device="cuda"), 0.25, 2.0)
    assert rel(yt.cpu().numpy(), OI.precond_mul(K, y2, x2, 0.25, 2.0)) <= 1e-13
    x6 = rng.standard_normal(6 * N)
    y6 = rng.standard_normal(6 * N)
    yt = torch.tensor(y6, device="cuda")
    kkt.mul(yt, torch.tensor(x6, device="cuda"), -1.0, 1.0)
    assert rel(yt.cpu().numpy(), OI.kkt_mul(ref, y6, x6, -1.0, 1.0)) <= 1e-12
    yt = torch.zeros(4 * N, dtype=torch.float64, device="cuda")
    kkt.jtprod(yt, torch.tensor(x2, device="cuda"))
    assert np.array_equal(yt.cpu().numpy(), OI.jtprod(x2, N))


@pytest.mark.parametrize("size", [(200,), (12, 18), (8, 6, 4)])
def test_kkt_solve(cuda, size):
    """solve_kkt! with Krylov.jl CG semantics (atol 1e-12, rtol 0)."""
    import csipm
    torch = cuda
    nlp, ref, z0, rng, N = setup(size, seed=4)
    kkt = csipm.FFTKKTSystem(nlp)
    pr = np.ones(4 * N)
    pr[2 * N:] = rng.uniform(0.1, 10.0, 2 * N)
    prt = torch.tensor(pr, device="cuda")
    kkt.build_kkt(prt)
    w = rng.standard_normal(6 * N)
    wt = torch.tensor(w, device="cuda")
    kkt.solve_kkt(wt, prt)
    sol_ref, it_ref = OI.kkt_solve(ref, OI.kkt_build(pr, N), w, pr, atol=1e-12, rtol=0.0)
    assert rel(wt.cpu().numpy(), sol_ref) <= 1e-9
    assert abs(kkt.krylov_iterations[-1] - it_ref) <= 1
