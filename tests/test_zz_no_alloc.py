"""csipm_apply_AtA_static — A^T A for callers that cannot allocate device
memory (a pool-owning runtime with a hard limit, a serving process that has
committed all HBM, a loop that cannot take cudaMalloc's synchronisation).  Its
scratch is a fixed 32 MiB device array shared by all calls.

Checked through the C ABI against the oracle (pocketfft, within the
operator's 1e-12) and against the handle-based csipm_apply_AtA, on calls in a
row of different sizes (each must not see the previous call's leftovers): 1D
rows on the one-CTA row pass and on the four-step long-row passes, masked 2D
and 3D grids, and lengths with odd factors (3, 5, 7, 11).  A second call
changes the device's free memory by nothing.  This file runs last."""
import ctypes

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12

# in call order: short 1D row, long 1D rows (four-step), masked 2D / 3D, odd factors, 1D again
SIZES = [(4096,), (16384,), (2 ** 16,), (24, 20, 16), (64, 48), (30, 42), (14, 22, 26), (2 * 3 * 5 * 7 * 11,),
         (96, 60, 50), (2 ** 20,), (1000,)]


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


def static_call(L, size, bits, x, y):
    import torch
    from csipm import _native
    n = (ctypes.c_int * 3)(*(list(size) + [1] * (3 - len(size))))
    st = L.csipm_apply_AtA_static(len(size), n, ctypes.c_void_p(bits.data_ptr()) if bits is not None else None,
                                  ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    _native.check(st)


def test_static_matches_oracle_and_handle(cuda):
    torch = cuda
    from csipm import _native
    L = _native.load()
    rng = np.random.default_rng(0)
    for size in SIZES:
        N = int(np.prod(size))
        keep = rng.random(N) > 0.15
        x_h = rng.standard_normal(N)
        x = torch.tensor(x_h, device="cuda")
        bits = torch.tensor(keep_bits(keep, size).view(np.int32), device="cuda")
        y = torch.full_like(x, float("nan"))
        static_call(L, size, bits, x, y)
        torch.cuda.synchronize()
        want = O.Operator(size, keep, True, workers=4).AtA(x_h)
        got = y.cpu().numpy()
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err <= TOL, (size, "oracle", err)
        y_ref = handle_AtA(size, keep, x)
        err = (torch.linalg.norm(y - y_ref) / torch.linalg.norm(y_ref)).item()
        assert err <= TOL, (size, "handle", err)


def test_static_allocates_nothing(cuda):
    """After a first call (the per-device set-up), further calls leave the
    device's free memory unchanged, and a call with no mask gives A^T A = I."""
    torch = cuda
    from csipm import _native
    L = _native.load()
    size = (64, 60, 40)
    N = int(np.prod(size))
    x = torch.randn(N, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    static_call(L, size, None, x, y)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        static_call(L, size, None, x, y)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert (torch.linalg.norm(y - x) / torch.linalg.norm(x)).item() <= TOL


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
