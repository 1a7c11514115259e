"""Data formats around the hot path, as the reference's benchmark drivers use
them (benchmarks/crystal.jl, benchmarks/mastodonte.jl):

* NPY volume input and the crystal punching: a 3D volume on a Cartesian grid
  x = x0 + dx*i, ..., cropped, with every grid point inside an ellipsoid of
  the given radius around each integer lattice point removed
  (crystal.jl:13-26 ``punch_3D_cart``, :29-98 ``crystal``);
* a 0/1 mask volume -> the 0-based column-major linear indices of the missing
  samples (mastodonte.jl:38-50);
* the recovered signal sqrt(N) * Re(IDFT(B beta)) from a solution
  (mastodonte.jl:109-116), written as NPY.

HDF5 input/output (mastodonte.jl:75-82, 114) needs h5py, which is not installed
here; ``read_h5_dataset`` / ``write_h5_dataset`` use it when present and raise
otherwise.
"""
from __future__ import annotations

import numpy as np


def read_npy(path):
    """A volume stored as NPY (npzread in the reference); indices (i, j, k) of
    the Julia array are numpy's [i, j, k]."""
    return np.load(path)


def punch_3D_cart(center, radius, x, y, z):
    """crystal.jl:13-26 with linear=true: the 0-based column-major linear
    indices of the grid points (x[i], y[j], z[k]) inside the ellipsoid of
    radii `radius` (a number or a 3-tuple) around `center`.  Raises on an
    empty punch, as the reference does."""
    rx, ry, rz = (radius if isinstance(radius, (tuple, list)) else (radius, radius, radius))
    x, y, z = (np.asarray(v, dtype=np.float64) for v in (x, y, z))
    dx = ((x - center[0]) / rx) ** 2
    dy = ((y - center[1]) / ry) ** 2
    dz = ((z - center[2]) / rz) ** 2
    inside = dx[:, None, None] + dy[None, :, None] + dz[None, None, :] <= 1.0
    idx = np.flatnonzero(inside.ravel(order="F"))
    if idx.size == 0:
        raise ValueError("Empty punch.")
    return idx


def crystal_grid(variant=True):
    """Grid, crop and lattice of crystal.jl:30-96 (variant: the punched_pmn
    volume, 310 x 410 x 410; else z3d_movo, 210 x 310 x 310)."""
    d = 0.02
    if variant:
        x, y, z = np.arange(-0.2, 6.01, d)[:310], np.arange(-0.2, 8.01, d)[:410], np.arange(-0.2, 8.01, d)[:410]
        lattice = (range(0, 7), range(0, 9), range(0, 9))
    else:
        x, y, z = np.arange(-0.2, 4.01, d)[:210], np.arange(-0.2, 6.01, d)[:310], np.arange(-0.2, 6.01, d)[:310]
        lattice = (range(0, 5), range(0, 7), range(0, 7))
    return x, y, z, lattice


def crystal_problem(z3d, variant=True, radius=0.2001, grid=None):
    """crystal.jl:29-98: crop the volume to the grid, punch every lattice
    point; returns (DFTsize, z0 flat column-major with zeros at the punches,
    0-based missing indices).  ``grid`` = (x, y, z, lattice) overrides the
    reference's grid (small volumes in tests)."""
    x, y, z, lattice = grid if grid is not None else crystal_grid(variant)
    size = (len(x), len(y), len(z))
    vol = np.asarray(z3d, dtype=np.float64)[:size[0], :size[1], :size[2]]
    missing = []
    for i in lattice[0]:
        for j in lattice[1]:
            for k in lattice[2]:
                missing.append(punch_3D_cart((float(i), float(j), float(k)), radius, x, y, z))
    missing = np.unique(np.concatenate(missing)).astype(np.int64)
    z0 = vol.ravel(order="F").copy()
    z0[missing] = 0.0
    return size, z0, missing


def mask_to_missing(mask):
    """mastodonte.jl:38-50: 0-based column-major linear indices where mask == 0."""
    return np.flatnonzero(np.asarray(mask).ravel(order="F") == 0).astype(np.int64)


def recover_signal(beta, DFTdim, DFTsize):
    """sqrt(N) * Re(IDFT(B beta)) on the device (the unmasked A of the
    library) — the write-back of mastodonte.jl:109-116.  beta: torch CUDA
    float64 tensor (N); returns a torch tensor (N, column-major)."""
    import torch
    from . import FFTOperator, FFTParameters
    n = int(np.prod(DFTsize))
    zeros = torch.zeros(n, dtype=torch.float64, device=beta.device)
    op = FFTOperator(FFTParameters(DFTdim, tuple(DFTsize), zeros, 0.0, None))
    try:
        return op.M_perp_beta(beta)
    finally:
        op.close()


def write_npy(path, x, DFTsize=None):
    """Writes a recovered signal as NPY, reshaped column-major to DFTsize when given."""
    a = x.detach().cpu().numpy() if hasattr(x, "detach") else np.asarray(x)
    if DFTsize is not None:
        a = a.reshape(tuple(DFTsize), order="F")
    np.save(path, a)


def _h5py():
    try:
        import h5py
    except ImportError as e:   # pragma: no cover - depends on the image
        raise RuntimeError("HDF5 I/O needs h5py, which is not installed") from e
    return h5py


def read_h5_dataset(path, name="data"):
    """read(h5open(path)[name]) of mastodonte.jl:75-82 (needs h5py)."""
    with _h5py().File(path, "r") as f:
        return np.asarray(f[name])


def write_h5_dataset(path, name, x):
    """h5write(path, name, x) of mastodonte.jl:114 (needs h5py)."""
    with _h5py().File(path, "w") as f:
        f[name] = np.asarray(x)
