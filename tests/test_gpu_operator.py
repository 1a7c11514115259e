"""A, A^T, A^T A on the GPU against the FP64 oracle (pocketfft), within 1e-12
relative (2-norm), on the reference's size grid and on larger / mixed-radix /
prime-factor grids, with and without missing samples."""
import numpy as np
import pytest

import oracle as O
from conftest import REF_GRID

pytestmark = pytest.mark.gpu

TOL = 1e-12
# 1D rows above 4096 samples take the multi-CTA four-step path (M = P*Q)
EXTRA = [(16384,), (1000,), (2 * 3 * 5 * 7 * 2,), (256, 256), (62, 82), (30, 42), (64, 64, 64), (32, 48, 40),
         (14, 22, 26), (20, 30, 18), (8192,), (4374,), (2 * 2 * 3 * 5 * 7 * 11,), (24000,), (65536,), (2 ** 20,)]
# every two-level factor pair of the strided passes (dims 2, 3) and of the
# row pass (dim 1: M = N1/2) that serves the 3D sides of 32-128 and the 2D
# sides of 128-1024 with factors 2, 3, 5
PAIR_GRID = [(120, 108, 80), (72, 72, 90), (108, 100, 96), (100, 40, 48), (64, 54, 36), (90, 60, 50),
             (80, 32, 120), (48, 96, 40), (96, 50, 54), (40, 36, 60), (60, 72, 32), (50, 90, 100), (120, 108),
             (90, 100), (360, 400), (960, 240), (450, 300), (600, 180), (360, 500), (960, 800), (32, 36, 40),
             (1024, 1024), (720, 864), (900, 432), (648, 960), (324, 576), (960, 900), (540, 600), (432, 324),
             (576, 360), (400, 810), (864, 256), (640, 128)]


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def make_op(size, keep, rdft=True):
    import csipm
    import torch
    N = int(np.prod(size))
    rng = np.random.default_rng(11)
    z0 = rng.standard_normal(N)
    if keep is not None:
        z0 = np.where(keep, z0, 0.0)
    params = csipm.FFTParameters(len(size), size, torch.tensor(z0, device="cuda"), 0.1,
                                 None if keep is None else np.flatnonzero(~keep))
    return csipm.FFTOperator(params, rdft=rdft), z0


@pytest.mark.parametrize("size", REF_GRID + EXTRA + PAIR_GRID)
@pytest.mark.parametrize("masked", [False, True])
def test_operator_matches_oracle(cuda, size, masked):
    torch = cuda
    N = int(np.prod(size))
    rng = np.random.default_rng(N + masked)
    keep = (rng.random(N) > 0.15) if masked else None
    op, z0 = make_op(size, keep)
    ref = O.Operator(size, keep)
    x = rng.standard_normal(N)
    xt = torch.tensor(x, device="cuda")
    assert relerr(op.M_perp_beta(xt).cpu().numpy(), ref.A(x)) <= TOL
    assert relerr(op.M_perpt_z(xt).cpu().numpy(), ref.At(x)) <= TOL
    assert relerr(op.M_perpt_M_perp_vec(xt).cpu().numpy(), ref.AtA(x)) <= TOL
    op.close()


@pytest.mark.parametrize("size", REF_GRID)
@pytest.mark.parametrize("rdft", [False, True])
def test_reference_unit_checks(cuda, size, rdft):
    """test/unit_tests_ipm.jl:21-30 on the GPU: A'A z = z with no mask, norms preserved."""
    torch = cuda
    N = int(np.prod(size))
    z = np.random.default_rng(0).random(N)
    op, _ = make_op(size, None, rdft)
    zt = torch.tensor(z, device="cuda")
    assert relerr(op.M_perpt_M_perp_vec(zt).cpu().numpy(), z) <= TOL
    assert abs(torch.linalg.norm(op.M_perpt_z(zt)).item() / np.linalg.norm(z) - 1) <= TOL
    assert abs(torch.linalg.norm(op.M_perp_beta(zt)).item() / np.linalg.norm(z) - 1) <= TOL
    op.close()


def test_adjointness_large_3d(cuda):
    """<A x, y> == <x, A^T y> at a production size (size-independent property)."""
    torch = cuda
    size = (160, 160, 160)
    N = int(np.prod(size))
    import csipm.problems as P
    keep = P.lattice_mask(size, 16, 3)
    op, _ = make_op(size, keep)
    g = torch.Generator("cuda").manual_seed(1)
    x = torch.randn(N, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(N, dtype=torch.float64, device="cuda", generator=g)
    y = y * torch.tensor(keep, device="cuda")
    lhs = torch.dot(op.M_perp_beta(x), y).item()
    rhs = torch.dot(x, op.M_perpt_z(y)).item()
    assert abs(lhs - rhs) <= 1e-11 * (abs(lhs) + 1e-300) * 100
    # A'A is a projection-like contraction: ||A'A x|| <= ||x||, and A'A x == A'(A x)
    q = op.M_perpt_M_perp_vec(x)
    q2 = op.M_perpt_z(op.M_perp_beta(x))
    assert (torch.linalg.norm(q - q2) / torch.linalg.norm(q)).item() <= TOL
    assert torch.linalg.norm(q).item() <= torch.linalg.norm(x).item() * (1 + 1e-12)
    op.close()
