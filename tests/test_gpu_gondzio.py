"""The Gondzio formulation on the device (csipm_gondzio_*, src/gondzio_model.jl
and src/gondzio_kkt.jl) against the CPU restatement oracle_gondzio.py."""
import numpy as np
import pytest

import oracle as O
import oracle_gondzio as OG

pytestmark = pytest.mark.gpu

SIZES = [(6000,), (48, 40), (16, 20, 12), (32, 64, 24)]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def _setup(torch, size, seed=3):
    import csipm
    rng = np.random.default_rng(seed)
    n = int(np.prod(size))
    keep = rng.random(n) > 0.15
    z0 = np.where(keep, rng.standard_normal(n), 0.0)
    lam = 0.3
    params = csipm.FFTParameters(len(size), size, torch.tensor(z0, device="cuda"), lam, np.flatnonzero(~keep))
    nlp = csipm.GondzioNLPModel(params, rdft=True)
    return rng, n, keep, z0, lam, nlp, O.Operator(size, keep), params


@pytest.mark.parametrize("size", SIZES)
def test_model_functions(cuda, size):
    torch = cuda
    rng, n, keep, z0, lam, nlp, op, params = _setup(torch, size)
    x = rng.standard_normal(3 * n)
    xt = torch.tensor(x, device="cuda")
    assert abs(nlp.obj(xt) - OG.obj(x, n, lam)) <= 1e-12 * abs(OG.obj(x, n, lam))
    g = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    assert np.array_equal(nlp.grad(xt, g).cpu().numpy(), OG.grad(x, n, lam))
    c = torch.empty(n, dtype=torch.float64, device="cuda")
    assert rel(nlp.cons(xt, c).cpu().numpy(), OG.cons(op, z0, x, n)) <= 1e-12
    nlp.op_fft.close()


@pytest.mark.parametrize("size", SIZES)
def test_kkt_products(cuda, size):
    import csipm
    torch = cuda
    rng, n, keep, z0, lam, nlp, op, params = _setup(torch, size)
    kkt = csipm.GondzioKKTSystem(nlp)
    pr = rng.uniform(0.05, 4.0, 3 * n)
    kkt.build_kkt(torch.tensor(pr, device="cuda"))
    K = OG.build(pr, n)
    x2 = rng.standard_normal(2 * n)
    y2 = rng.standard_normal(2 * n)
    a, b = 0.7, -0.4
    yt = torch.tensor(y2, device="cuda")
    kkt.condensed_mul(yt, torch.tensor(x2, device="cuda"), a, b)
    assert rel(yt.cpu().numpy(), a * OG.condensed_mul(op, K, x2, n) + b * y2) <= 1e-12
    yt = torch.tensor(y2, device="cuda")
    kkt.precond_mul(yt, torch.tensor(x2, device="cuda"), a, b)
    assert rel(yt.cpu().numpy(), a * OG.precond_mul(K, x2, n) + b * y2) <= 1e-13
    x4 = rng.standard_normal(4 * n)
    y4 = rng.standard_normal(4 * n)
    yt = torch.tensor(y4, device="cuda")
    kkt.mul(yt, torch.tensor(x4, device="cuda"), a, b)
    assert rel(yt.cpu().numpy(), OG.kkt_mul_body(op, x4, n, a, b, y4)) <= 1e-12
    xn = rng.standard_normal(n)
    yt = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    kkt.jtprod(yt, torch.tensor(xn, device="cuda"))
    assert rel(yt.cpu().numpy(), OG.jtprod(op, xn, n)) <= 1e-12
    nlp.op_fft.close()


@pytest.mark.parametrize("size", SIZES)
def test_kkt_solve(cuda, size):
    """Same PCG (block preconditioner, atol 1e-12, rtol 0): the solution within
    1e-9 relative of the CPU solve and the iteration count within 2."""
    import csipm
    torch = cuda
    rng, n, keep, z0, lam, nlp, op, params = _setup(torch, size)
    kkt = csipm.GondzioKKTSystem(nlp)
    pr = rng.uniform(0.05, 4.0, 3 * n)
    kkt.build_kkt(torch.tensor(pr, device="cuda"))
    K = OG.build(pr, n)
    w = rng.standard_normal(4 * n)
    wt = torch.tensor(w, device="cuda")
    kkt.solve_kkt(wt)
    ref, it = OG.kkt_solve(op, K, w, n)
    assert rel(wt.cpu().numpy(), ref) <= 1e-9
    assert abs(kkt.krylov_iterations[-1] - it) <= 2
    nlp.op_fft.close()
