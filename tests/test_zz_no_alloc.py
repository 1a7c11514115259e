"""csipm_apply_AtA_static — A^T A for callers that cannot allocate device
memory (a pool-owning runtime with a hard limit, a serving process that has
committed all HBM, a loop that cannot take cudaMalloc's synchronisation).  Its
scratch is a fixed 32 MiB device array shared by all calls.  Checked through
the C ABI against the handle-based csipm_apply_AtA, on two calls in a row of
different sizes (the second must not see the first's leftovers)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def keep_bits(keep, size):
    """Row-padded bitmask: one bit per sample (1 = observed), column-major,
    LSB first, each dim-1 row of N1 bits padded to 32-bit words."""
    n1 = size[0]
    rows = int(np.prod(size[1:])) if len(size) > 1 else 1
    wpr = (n1 + 31) // 32
    k = keep.reshape(rows, n1)
    padded = np.zeros((rows, wpr * 32), dtype=np.uint8)
    padded[:, :n1] = k
    bits = np.packbits(padded.reshape(rows, wpr, 32), axis=2, bitorder="little")
    return np.ascontiguousarray(bits).view(np.uint32).reshape(-1)


def handle_AtA(size, keep, x):
    import csipm
    import torch
    params = csipm.FFTParameters(len(size), size, torch.zeros(int(np.prod(size)), dtype=torch.float64, device="cuda"),
                                 0.0, np.flatnonzero(~keep))
    op = csipm.FFTOperator(params)
    y = op.M_perpt_M_perp_vec(x).clone()
    op.close()
    return y


def static_AtA(size, keep, x):
    import torch
    from csipm import _native
    L = _native.load()
    y = torch.full_like(x, float("nan"))
    bits = torch.tensor(keep_bits(keep, size).view(np.int32), device="cuda") if keep is not None else None
    n = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - len(size))))
    st = L.csipm_apply_AtA_static(len(size), n, ctypes.c_void_p(bits.data_ptr()) if bits is not None else None,
                                  ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _native.check(st)
    torch.cuda.synchronize()
    return y


def test_static_matches_handle_two_calls(cuda):
    torch = cuda
    rng = np.random.default_rng(0)
    for size in [(24, 20, 16), (64, 48)]:          # two calls in a row, different sizes
        N = int(np.prod(size))
        keep = rng.random(N) > 0.15
        x = torch.tensor(rng.standard_normal(N), device="cuda")
        y_static = static_AtA(size, keep, x)
        y_ref = handle_AtA(size, keep, x)
        err = (torch.linalg.norm(y_static - y_ref) / torch.linalg.norm(y_ref)).item()
        assert err <= TOL, (size, err)


def test_static_rejects_oversize(cuda):
    torch = cuda
    from csipm import _native
    L = _native.load()
    size = (2048, 2048)
    x = torch.zeros(size[0] * size[1], dtype=torch.float64, device="cuda")
    n = (ctypes.c_int * 3)(size[0], size[1], 1)
    st = L.csipm_apply_AtA_static(2, n, None, ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(x.data_ptr()), None)
    assert st == _native.CSIPM_ERR_UNSUPPORTED
    assert b"32 MiB" in L.csipm_last_error(None)
