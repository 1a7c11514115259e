"""Data formats of the reference's benchmark drivers (csipm.io): crystal
punching (benchmarks/crystal.jl), mask volumes (benchmarks/mastodonte.jl) and
the recovered-signal write-back."""
import os

import numpy as np
import pytest

import oracle as O


def test_punch_matches_brute_force():
    from csipm.io import punch_3D_cart
    x = np.arange(-0.2, 1.21, 0.1)[:14]
    y = np.arange(-0.2, 1.61, 0.1)[:18]
    z = np.arange(-0.2, 1.01, 0.1)[:12]
    got = punch_3D_cart((1.0, 1.0, 0.0), (0.25, 0.31, 0.2), x, y, z)
    want = []
    for k in range(len(z)):
        for j in range(len(y)):
            for i in range(len(x)):
                if ((x[i] - 1) / 0.25) ** 2 + ((y[j] - 1) / 0.31) ** 2 + ((z[k] - 0) / 0.2) ** 2 <= 1.0:
                    want.append(i + len(x) * (j + len(y) * k))
    assert got.tolist() == want
    with pytest.raises(ValueError):
        punch_3D_cart((10.0, 10.0, 10.0), 0.01, x, y, z)


def test_crystal_problem_small_grid():
    from csipm.io import crystal_problem
    d = 0.05
    grid = (np.arange(-0.2, 1.31, d)[:30], np.arange(-0.2, 1.31, d)[:30], np.arange(-0.2, 1.31, d)[:30],
            (range(0, 2), range(0, 2), range(0, 2)))
    vol = np.random.default_rng(0).standard_normal((32, 32, 32))
    size, z0, missing = crystal_problem(vol, radius=0.2001, grid=grid)
    assert size == (30, 30, 30)
    assert missing.size > 0 and np.all(z0[missing] == 0.0)
    keep = np.ones(z0.size, bool)
    keep[missing] = False
    assert np.array_equal(z0[keep], vol[:30, :30, :30].ravel(order="F")[keep])


def test_mask_to_missing_column_major():
    from csipm.io import mask_to_missing
    m = np.ones((4, 3, 2))
    m[1, 2, 0] = 0
    m[3, 0, 1] = 0
    assert mask_to_missing(m).tolist() == [1 + 4 * 2, 3 + 4 * 3 * 1]


def test_npy_round_trip(tmp_path):
    from csipm.io import read_npy, write_npy
    x = np.arange(24.0)
    write_npy(os.path.join(tmp_path, "s.npy"), x, (2, 3, 4))
    y = read_npy(os.path.join(tmp_path, "s.npy"))
    assert y.shape == (2, 3, 4) and np.array_equal(y.ravel(order="F"), x)


@pytest.mark.gpu
def test_recover_signal_and_solve(cuda, tmp_path):
    """A crystal-style punched volume through the whole path: recover beta,
    write sqrt(N) Re(IDFT(B beta)) back, and compare that with the oracle's
    unmasked A."""
    import csipm
    from csipm.io import crystal_problem, recover_signal, write_npy, read_npy
    torch = cuda
    d = 0.05
    grid = (np.arange(-0.2, 1.91, d)[:40], np.arange(-0.2, 1.91, d)[:40], np.arange(-0.2, 1.31, d)[:24],
            (range(0, 2), range(0, 2), range(0, 2)))
    rng = np.random.default_rng(1)
    size = (40, 40, 24)
    beta_true = np.zeros(int(np.prod(size)))
    beta_true[rng.choice(beta_true.size, 300, replace=False)] = rng.standard_normal(300)
    vol = O.Operator(size).A(beta_true).reshape(size, order="F")
    size, z0, missing = crystal_problem(vol, radius=0.2001, grid=grid)
    params = csipm.FFTParameters(3, size, torch.tensor(z0, device="cuda"), 0.01, missing)
    res = csipm.ipm_solve(csipm.FFTNLPModel(params, rdft=True))
    assert res.status == 0
    x = recover_signal(res.beta, 3, size)
    ref = O.Operator(size).A(res.beta.cpu().numpy())
    assert np.linalg.norm(x.cpu().numpy() - ref) <= 1e-12 * np.linalg.norm(ref)
    p = os.path.join(tmp_path, "solution.npy")
    write_npy(p, x, size)
    assert np.allclose(read_npy(p).ravel(order="F"), ref, rtol=0, atol=1e-10 * np.abs(ref).max())
