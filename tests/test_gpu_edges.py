"""Edge cases on the device: the smallest grids, duplicate and out-of-range
missing indices, every sample of a row missing, and lambda above ||A'z0||_inf
(where beta = 0 is the LASSO optimum)."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("size", [(2,), (4,), (2, 2), (2, 6), (4, 2), (2, 2, 2), (2, 2, 4), (4, 2, 2)])
def test_smallest_grids_match_oracle(cuda, size):
    import csipm
    torch = cuda
    N = int(np.prod(size))
    rng = np.random.default_rng(N)
    keep = rng.random(N) > 0.3
    z0 = np.where(keep, rng.standard_normal(N), 0.0)
    params = csipm.FFTParameters(len(size), size, torch.tensor(z0, device="cuda"), 0.1, np.flatnonzero(~keep))
    op = csipm.FFTOperator(params)
    ref = O.Operator(size, keep)
    x = rng.standard_normal(N)
    xt = torch.tensor(x, device="cuda")
    assert rel(op.M_perp_beta(xt).cpu().numpy(), ref.A(x)) <= 1e-12
    assert rel(op.M_perpt_z(xt).cpu().numpy(), ref.At(x)) <= 1e-12
    assert rel(op.M_perpt_M_perp_vec(xt).cpu().numpy(), ref.AtA(x)) <= 1e-12
    op.close()


def test_duplicate_missing_indices_change_nothing(cuda):
    import csipm
    torch = cuda
    size = (24, 20)
    N = 24 * 20
    rng = np.random.default_rng(5)
    miss = rng.choice(N, 60, replace=False)
    z0 = rng.standard_normal(N)
    z0[miss] = 0.0
    x = torch.tensor(rng.standard_normal(N), device="cuda")
    out = []
    for m in (miss, np.concatenate([miss, miss[:20]])):
        op = csipm.FFTOperator(csipm.FFTParameters(2, size, torch.tensor(z0, device="cuda"), 0.1, m))
        out.append(op.M_perpt_M_perp_vec(x).cpu().numpy())
        op.close()
    assert np.array_equal(out[0], out[1])


def test_out_of_range_missing_index_is_rejected(cuda):
    import csipm
    from csipm import _native
    torch = cuda
    size = (16, 16)
    with pytest.raises(_native.CsipmError) as e:
        csipm.FFTOperator(csipm.FFTParameters(2, size, torch.zeros(256, dtype=torch.float64, device="cuda"), 0.1,
                                              np.array([3, 256])))
    assert e.value.status == _native.CSIPM_ERR_INVALID


def test_fully_missing_row(cuda):
    """Every sample of one dim-1 row missing (a whole mask word run cleared)."""
    import csipm
    torch = cuda
    size = (64, 8)
    N = 512
    keep = np.ones(N, bool)
    keep[64 * 3:64 * 4] = False
    rng = np.random.default_rng(2)
    z0 = np.where(keep, rng.standard_normal(N), 0.0)
    op = csipm.FFTOperator(csipm.FFTParameters(2, size, torch.tensor(z0, device="cuda"), 0.1, np.flatnonzero(~keep)))
    x = rng.standard_normal(N)
    assert rel(op.M_perpt_M_perp_vec(torch.tensor(x, device="cuda")).cpu().numpy(), O.Operator(size, keep).AtA(x)) <= 1e-12
    op.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_large_lambda_gives_zero(cuda, precision):
    """lambda >= ||A'z0||_inf: beta = 0 is optimal, F = 1/2 ||z0||^2."""
    import csipm
    torch = cuda
    size = (32, 24)
    N = 32 * 24
    rng = np.random.default_rng(4)
    keep = rng.random(N) > 0.1
    z0 = np.where(keep, rng.standard_normal(N), 0.0)
    lam = 2.0 * np.abs(O.Operator(size, keep).At(z0)).max()
    params = csipm.FFTParameters(2, size, torch.tensor(z0, device="cuda"), lam, np.flatnonzero(~keep))
    res = csipm.ipm_solve(csipm.FFTNLPModel(params, rdft=True, precision=precision, tol=1e-10))
    assert res.status == 0, res.stats
    assert np.abs(res.beta.cpu().numpy()).max() <= 1e-6 * np.abs(z0).max()
    assert abs(res.stats["lasso_obj"] - 0.5 * float(z0 @ z0)) <= 1e-8 * 0.5 * float(z0 @ z0)
