"""beta <-> DFT map kernels on the GPU: bit-exact with the oracle's restatement
of src/mapping_cpu_kernels.jl (including signed zeros), half and full spectra."""
import numpy as np
import pytest

import oracle as O
from conftest import REF_GRID

pytestmark = pytest.mark.gpu

SIZES = REF_GRID + [(2,), (4,), (2, 2), (2, 6), (6, 2), (2, 2, 2), (4, 2, 6), (320,), (30, 50), (10, 14, 22)]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("size", SIZES)
@pytest.mark.parametrize("rdft", [True, False])
@pytest.mark.parametrize("zeros", [False, True])
def test_beta_to_dft_bit_exact(cuda, size, rdft, zeros):
    import csipm
    torch = cuda
    rng = np.random.default_rng(abs(hash((size, rdft, zeros))) % 2 ** 32)
    N = int(np.prod(size))
    beta = rng.choice([-0.0, 0.0, 1.25, -3.5], size=N) if zeros else rng.standard_normal(N)
    v = csipm.beta_to_DFT(len(size), size, torch.tensor(beta, device="cuda"), rdft=rdft)
    ref = O.beta_to_dft(beta, size, rdft, "kern")
    got = v.cpu().numpy()
    assert got.shape == ref.shape
    assert np.array_equal(_bits(got.ravel(order="F").view(np.float64)), _bits(np.asfortranarray(ref).ravel(order="F").view(np.float64)))


@pytest.mark.parametrize("size", SIZES)
@pytest.mark.parametrize("full", [False, True])
def test_dft_to_beta_bit_exact(cuda, size, full):
    import csipm
    torch = cuda
    rng = np.random.default_rng(abs(hash((size, full))) % 2 ** 32)
    shp = size if full else (size[0] // 2 + 1,) + tuple(size[1:])
    v = np.asfortranarray(rng.standard_normal(shp) + 1j * rng.standard_normal(shp))
    vt = torch.tensor(np.ascontiguousarray(v.transpose(*reversed(range(v.ndim)))), device="cuda")
    vt = vt.permute(*reversed(range(v.ndim)))
    beta = csipm.DFT_to_beta(len(size), size, vt).cpu().numpy()
    ref = O.dft_to_beta(v, size, "kern")
    assert np.array_equal(_bits(beta), _bits(ref))


def test_maps_large_3d_roundtrip(cuda):
    """At a production size the maps are checked through a size-independent
    property: DFT_to_beta(beta_to_DFT(beta)) == beta up to one rounding."""
    import csipm
    torch = cuda
    size = (128, 96, 64)
    beta = torch.randn(int(np.prod(size)), dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(0))
    v = csipm.beta_to_DFT(3, size, beta, rdft=True)
    back = csipm.DFT_to_beta(3, size, v)
    assert torch.allclose(back, beta, rtol=5e-16, atol=0)


def test_odd_dimension_rejected(cuda):
    import csipm
    torch = cuda
    with pytest.raises(ValueError):
        csipm.beta_to_DFT(2, (5, 4), torch.zeros(20, dtype=torch.float64, device="cuda"))
