"""Batched solves (csipm_solve_batch): recoveries of uneven sizes advanced
together, every step one kernel launch for all of them (instance table with
per-instance sizes, plans and vector offsets).  Each instance must reach the
optimum csipm_solve reaches alone and the CPU twin's: beta within 1e-6
relative, objective within 1e-8 relative, IPM iterations within 1."""
import numpy as np
import pytest

import oracle as O
import oracle_ipm as OI

pytestmark = pytest.mark.gpu


def _problem(kind, dims, seed):
    import csipm.problems as P
    spec = P.make_spec(kind, dims=dims, seed=seed)
    op0 = O.Operator(spec.size)
    return P.finalize(spec, op0.A, op0.At)


def _model(torch, prob, **kw):
    import csipm
    size = prob.size
    params = csipm.FFTParameters(len(size), size, torch.tensor(prob.z0, device="cuda"), prob.lam, prob.missing)
    return csipm.FFTNLPModel(params, rdft=True, **kw)


BATCHES = {
    "2d": [("2d", (64, 64)), ("2d", (128, 96)), ("2d", (96, 128)), ("2d", (200, 160)), ("2d", (48, 90))],
    "3d": [("3d", (16, 16, 16)), ("3d", (32, 64, 24)), ("3d", (48, 40, 36)), ("3d", (32, 32, 32))],
    "1d": [("1d", (2048,)), ("1d", (1000,)), ("1d", (4096,)), ("1d", (3000,))],
    "1d-long": [("1d", (16384,)), ("1d", (8192,)), ("1d", (24000,)), ("1d", (65536,))],
}


@pytest.mark.parametrize("group", sorted(BATCHES))
def test_batch_matches_single_and_twin(cuda, group):
    import csipm
    torch = cuda
    probs = [_problem(kind, dims, seed=30 + k) for k, (kind, dims) in enumerate(BATCHES[group])]
    opts = dict(tol=1e-10, ipm_cg_rtol=1e-2)
    batch = csipm.ipm_solve_batch([_model(torch, p, **opts) for p in probs])
    for prob, res in zip(probs, batch):
        assert res.status == 0, res.stats
        alone = csipm.ipm_solve(_model(torch, prob, **opts))
        assert alone.status == 0
        bb, ba = res.beta.cpu().numpy(), alone.beta.cpu().numpy()
        assert np.linalg.norm(bb - ba) / np.linalg.norm(ba) <= 1e-6
        assert abs(res.stats["ipm_iter"] - alone.stats["ipm_iter"]) <= 1
        op = O.Operator(prob.size, prob.spec.keep)
        b = op.At(prob.z0)
        beta, _, info = OI.ipm(op, b, prob.lam, float(prob.z0 @ prob.z0), tol=1e-10, cg_rtol=1e-2)
        assert np.linalg.norm(bb - beta) / np.linalg.norm(beta) <= 1e-6
        Fb = OI.lasso_value(op, bb, prob.z0, prob.lam)
        Fc = OI.lasso_value(op, beta, prob.z0, prob.lam)
        assert abs(Fb - Fc) <= 1e-8 * abs(Fc)
        assert abs(res.stats["ipm_iter"] - info["ipm_iter"]) <= 1


def test_batch_instances_stop_on_their_own(cuda):
    """An instance capped at 2 iterations stops there (status max_iter) while
    the others of its batch run to convergence."""
    import csipm
    from csipm import _native
    torch = cuda
    probs = [_problem("2d", (64, 64), seed=41), _problem("2d", (96, 80), seed=42), _problem("2d", (64, 96), seed=43)]
    models = [_model(torch, probs[0], tol=1e-10, ipm_cg_rtol=1e-2, max_iter=2),
              _model(torch, probs[1], tol=1e-10, ipm_cg_rtol=1e-2),
              _model(torch, probs[2], tol=1e-8, ipm_cg_rtol=1e-3)]
    batch = csipm.ipm_solve_batch(models)
    assert batch[0].status == _native.CSIPM_ERR_IPM_MAXITER and batch[0].stats["ipm_iter"] == 2
    for k in (1, 2):
        assert batch[k].status == 0
        alone = csipm.ipm_solve(_model(torch, probs[k], **({"tol": 1e-10, "ipm_cg_rtol": 1e-2} if k == 1 else
                                                          {"tol": 1e-8, "ipm_cg_rtol": 1e-3})))
        rel = np.linalg.norm(batch[k].beta.cpu().numpy() - alone.beta.cpu().numpy()) / np.linalg.norm(
            alone.beta.cpu().numpy())
        assert rel <= 1e-6


def test_batch_rejects_mixed_kinds(cuda):
    import csipm
    from csipm import _native
    torch = cuda
    m2 = _model(torch, _problem("2d", (64, 64), seed=1))
    m3 = _model(torch, _problem("3d", (16, 16, 16), seed=1))
    with pytest.raises(_native.CsipmError) as e:
        csipm.ipm_solve_batch([m2, m3])
    assert e.value.status == _native.CSIPM_ERR_INVALID


def test_batch_takes_mixed_precision_handles(cuda):
    """Handles created for mixed precision join a batch and are solved on its
    FP64 path: each result equals the FP64 solve alone (beta within 1e-6)."""
    import csipm
    torch = cuda
    probs = [_problem("3d", (32, 32, 32), seed=51), _problem("3d", (40, 36, 48), seed=52)]
    opts = dict(tol=1e-10, ipm_cg_rtol=1e-2)
    batch = csipm.ipm_solve_batch([_model(torch, p, precision="mixed", **opts) for p in probs])
    for prob, res in zip(probs, batch):
        assert res.status == 0, res.stats
        alone = csipm.ipm_solve(_model(torch, prob, precision="fp64", **opts))
        b, a = res.beta.cpu().numpy(), alone.beta.cpu().numpy()
        assert np.linalg.norm(b - a) / np.linalg.norm(a) <= 1e-6
