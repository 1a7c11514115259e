"""The Gondzio restatement (oracle/oracle_gondzio.py): its KKT solve satisfies
the reduced system it stands for (gondzio_kkt.jl:318-332), and its products
agree with their definitions."""
import numpy as np

import oracle as O
import oracle_gondzio as OG


def _setup(size=(24, 20), seed=1):
    rng = np.random.default_rng(seed)
    n = int(np.prod(size))
    keep = rng.random(n) > 0.2
    op = O.Operator(size, keep)
    pr = rng.uniform(0.1, 5.0, 3 * n)
    return rng, n, op, pr


def test_kkt_solve_satisfies_reduced_system():
    rng, n, op, pr = _setup()
    K = OG.build(pr, n)
    w = rng.standard_normal(4 * n)
    sol, it = OG.kkt_solve(op, K, w, n)
    dx, dr, dy = sol[:2 * n], sol[2 * n:3 * n], sol[3 * n:]
    # [ D  0 -U'] [dx]   [r1]     U x = A(p - q)
    # [ 0  I -I ] [dr] = [r2]
    # [-U -I  0 ] [dy]   [r3]
    Ut_dy = np.concatenate([op.At(dy), -op.At(dy)])
    r1 = np.concatenate([K[0], K[1]]) * dx - Ut_dy
    assert np.linalg.norm(r1 - w[:2 * n]) <= 1e-9 * np.linalg.norm(w)
    assert np.allclose(dr - dy, w[2 * n:3 * n], atol=1e-12)
    assert np.allclose(-op.A(dx[:n] - dx[n:]) - dr, w[3 * n:], atol=1e-12)
    assert 0 < it <= 4 * n


def test_preconditioner_inverts_identity_model():
    """With A'A replaced by I the block preconditioner is the exact inverse."""
    rng, n, op, pr = _setup()
    K = OG.build(pr, n)
    x = rng.standard_normal(2 * n)
    Kx = np.concatenate([K[0] * x[:n] + x[:n] - x[n:], K[1] * x[n:] - (x[:n] - x[n:])])
    assert np.allclose(OG.precond_mul(K, Kx, n), x, rtol=0, atol=1e-12)
