"""The oracle's three statements of the beta <-> DFT packing agree (CPU)."""
import numpy as np
import pytest

import oracle as O
from conftest import REF_GRID

SIZES = REF_GRID + [(2,), (4,), (2, 2), (2, 6), (6, 2), (2, 2, 2), (4, 2, 6)]


def _bits(v):
    return np.ascontiguousarray(np.asarray(v).ravel(order="F")).view(np.uint64)


@pytest.mark.parametrize("size", SIZES)
@pytest.mark.parametrize("rdft", [True, False])
def test_kern_loops_wei_agree(size, rdft):
    rng = np.random.default_rng(hash(size) % 2 ** 32)
    beta = rng.standard_normal(int(np.prod(size)))
    vk = O.beta_to_dft(beta, size, rdft, "kern")
    vl = O.beta_to_dft(beta, size, rdft, "loops")
    vw = O.beta_to_dft(beta, size, rdft, "wei")
    assert not np.isnan(vk).any() and not np.isnan(vl).any()
    # mapping_cpu.jl and mapping_cpu_kernels.jl agree bit for bit on generic data
    assert np.array_equal(_bits(vk), _bits(vl))
    assert np.array_equal(vk, vw)
    for impl in ("kern", "loops"):
        # (b/sqrt2)*sqrt2 is within one rounding of b
        assert np.allclose(O.dft_to_beta(vk, size, impl), beta, rtol=5e-16, atol=0)


@pytest.mark.parametrize("size", [(16,), (12, 18), (6, 10, 12)])
def test_signed_zero_rules(size):
    """With +-0 entries the files differ only in the sign of zeros on conj mirrors;
    all statements stay equal as values."""
    rng = np.random.default_rng(7)
    beta = rng.choice([-0.0, 0.0, 1.0, -2.0], size=int(np.prod(size)))
    for rdft in (True, False):
        vk = O.beta_to_dft(beta, size, rdft, "kern")
        vl = O.beta_to_dft(beta, size, rdft, "loops")
        assert np.array_equal(vk, vl)


def test_hand_derived_1d():
    """src/mapping_cpu.jl:189-204 for N=4: v = [b1, (b3 + i b4)/sqrt2, b2 | (b3 - i b4)/sqrt2]."""
    b = np.array([1.5, -2.0, 3.0, 4.0])
    s2 = np.sqrt(2.0)
    v = O.beta_to_dft(b, (4,), rdft=False)
    assert np.array_equal(v, np.array([1.5, (3 + 4j) / s2, -2.0, (3 - 4j) / s2]))
    assert np.allclose(O.dft_to_beta(v, (4,)), b, rtol=5e-16, atol=0)


def test_hand_derived_2d_vertices():
    """src/mapping_cpu.jl:22-25: the four real vertices come first."""
    size = (4, 6)
    rng = np.random.default_rng(1)
    beta = rng.standard_normal(24)
    v = O.beta_to_dft(beta, size, rdft=True)
    assert v[0, 0] == beta[0] and v[0, 3] == beta[1] and v[2, 0] == beta[2] and v[2, 3] == beta[3]


@pytest.mark.parametrize("size", SIZES)
def test_full_spectrum_is_hermitian(size):
    rng = np.random.default_rng(3)
    beta = rng.standard_normal(int(np.prod(size)))
    v = O.beta_to_dft(beta, size, rdft=False)
    idx = tuple((-np.arange(n)) % n for n in size)
    mirror = v[np.ix_(*idx)]
    assert np.allclose(v, np.conj(mirror), rtol=0, atol=1e-15)
