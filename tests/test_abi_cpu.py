"""The C-ABI library loads and exports every symbol include/csipm.h declares (no GPU calls)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "csipm.h")).read()
    return sorted(set(re.findall(r"CSIPM_API\s+[\w\s\*]+?\b(csipm_\w+)\s*\(", hdr)))


def test_header_declares_expected_surface():
    from csipm import _native
    assert set(declared_symbols()) == set(_native.EXPORTS)


def test_library_exports_every_declared_symbol():
    from csipm import _native
    if not os.path.exists(_native.LIB_PATH):
        pytest.fail("libcsipm.so is not built (run __graft_entry__.build())")
    lib = ctypes.CDLL(_native.LIB_PATH)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_default_options_without_gpu():
    from csipm import _native
    L = _native.load()
    o = _native.Options()
    assert L.csipm_default_options(ctypes.byref(o)) == 0
    assert o.rdft == 1 and o.tol == 1e-8 and o.max_iter == 2000 and o.cg_atol == 1e-12 and o.cg_rtol == 0.0


def test_invalid_sizes_rejected_without_gpu():
    """Odd dimensions are rejected before any device work (src/fft_utils.jl requires even sizes)."""
    from csipm import _native
    L = _native.load()
    n = (ctypes.c_int * 3)(5, 4, 1)
    st = L.csipm_beta_to_dft(2, n, 1, None, None, None)
    assert st == _native.CSIPM_ERR_ODD_DIM
    assert b"even" in L.csipm_last_error(None)


def test_size_limits_and_footprint_without_gpu():
    """N >= 2^31 is refused (32-bit indices on the device); csipm_footprint is
    host arithmetic: it grows with the size and with mixed precision."""
    from csipm import _native
    L = _native.load()
    big = (ctypes.c_int * 3)(2048, 2048, 1024)
    out = ctypes.c_size_t()
    assert L.csipm_footprint(3, big, 0, 0, ctypes.byref(out)) == _native.CSIPM_ERR_UNSUPPORTED
    small = (ctypes.c_int * 3)(64, 64, 64)
    mid = (ctypes.c_int * 3)(128, 128, 128)
    f = []
    for size, prec in ((small, 0), (mid, 0), (mid, 1)):
        assert L.csipm_footprint(3, size, prec, 0, ctypes.byref(out)) == 0
        f.append(out.value)
    assert f[0] < f[1] < f[2]
    assert f[1] >= 26 * 8 * 128 ** 3   # 24 FP64 vectors + the server's z0/beta staging


def test_options_defaults_of_the_later_fields():
    from csipm import _native
    L = _native.load()
    o = _native.Options()
    assert L.csipm_default_options(ctypes.byref(o)) == 0
    assert o.layout == 0 and o.cuda_graphs == 1 and o.autotune == 1 and o.precision == 0
