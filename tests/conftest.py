import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "compressedsensingipm.jl_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

# The size grid of the reference's operator unit tests (test/unit_tests_ipm.jl:4, 80, 155).
SIZES_1D = [(100,), (200,), (500,)]
SIZES_2D = [(16, 16), (12, 18), (16, 24), (32, 32)]
SIZES_3D = [(8, 8, 8), (2, 4, 6), (6, 10, 12), (14, 8, 4), (8, 6, 4), (16, 16, 16)]
REF_GRID = SIZES_1D + SIZES_2D + SIZES_3D


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libcsipm.so")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import csipm
    csipm.lib()          # raises if the extension is missing: no fallback
    return torch
