"""Seeded synthetic recovery problems with the shapes, sparsities, masks, noise
levels and lambda rules of the workloads this library is measured on.

There is no public dataset for this path: the crystallography volumes used by
the reference's benchmarks (benchmarks/crystal.jl, benchmarks/mastodonte.jl)
are not available, so these generators stand in for them.

A problem is built in two steps so that the synthesis can run on whichever
operator the caller has (the CUDA library on a GPU, anything else in tests):

    spec = make_spec("3d", n=256, seed=0)          # beta_true, keep-mask, noise
    prob = finalize(spec, synth)                   # synth(beta) = A_full beta

``synth`` must apply the unmasked synthesis sqrt(N) * Re(IDFT(B beta)).
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class ProblemSpec:
    name: str
    size: tuple
    beta_true: np.ndarray          # float64, length N (beta <-> DFT packing order)
    keep: np.ndarray               # bool, length N, column-major; True = observed
    noise: np.ndarray              # float64, length N
    lam_factor: float              # lambda = lam_factor * ||A^T y||_inf
    seed: int

    @property
    def N(self):
        return int(np.prod(self.size))

    @property
    def n_missing(self):
        return int(self.N - self.keep.sum())


@dataclasses.dataclass
class Problem:
    spec: ProblemSpec
    z0: np.ndarray                 # observed signal, zero at missing samples
    lam: float
    missing: np.ndarray            # int64 0-based linear indices (column-major) of missing samples

    @property
    def size(self):
        return self.spec.size

    @property
    def N(self):
        return self.spec.N


def _sparse_beta(rng, N, frac, lognormal=False):
    k = max(1, int(round(frac * N)))
    idx = rng.choice(N, size=k, replace=False)
    beta = np.zeros(N)
    if lognormal:
        mag = rng.lognormal(0.0, 1.0, size=k)
        sgn = rng.choice([-1.0, 1.0], size=k)
        beta[idx] = mag * sgn
    else:
        beta[idx] = rng.standard_normal(k)
    return beta


def gap_mask_1d(rng, N, frac, ngaps):
    """ngaps random contiguous gaps that together remove round(frac*N) samples."""
    total = int(round(frac * N))
    cuts = np.sort(rng.choice(np.arange(1, total), size=ngaps - 1, replace=False))
    lengths = np.diff(np.concatenate([[0], cuts, [total]]))
    free = N - total
    spc = np.sort(rng.choice(np.arange(free + 1), size=ngaps, replace=True))
    keep = np.ones(N, dtype=bool)
    pos = 0
    prev = 0
    for g in range(ngaps):
        pos += spc[g] - prev
        prev = spc[g]
        keep[pos:pos + lengths[g]] = False
        pos += lengths[g]
    return keep


def lattice_mask(size, period, radius, offset=None):
    """Punch Euclidean balls of `radius` around every lattice point of `period`
    (Bragg-peak removal).  Column-major keep-mask."""
    size = tuple(size)
    if offset is None:
        offset = period // 2
    grids = np.meshgrid(*[np.arange(n) for n in size], indexing="ij")
    d2 = np.zeros(size)
    for g in grids:
        r = (g - offset) % period
        r = np.minimum(r, period - r)
        d2 = d2 + r.astype(np.float64) ** 2
    keep = d2 > radius * radius
    return keep.ravel(order="F")


def make_spec(kind, n=None, seed=0, dims=None):
    """The measured workloads:

    * "1d":  N=2^14, 2% N(0,1) nonzeros, 20 gaps removing 15%, sigma=0.01, lambda=0.1||A^T y||_inf
    * "2d":  1024^2, 1% N(0,1), disks r=4 on a period-32 lattice + 5% random pixels,
             sigma=0.01, lambda=0.1||A^T y||_inf
    * "3d":  n^3 (256 or 320), 0.5% log-normal(0,1) magnitudes with random signs,
             balls r=3 on a period-16 lattice (~3% missing), sigma=0.01,
             lambda=0.05||A^T y||_inf
    ``dims`` overrides the grid (every dimension must be even).
    """
    rng = np.random.default_rng(seed)
    if kind == "1d":
        size = tuple(dims) if dims else ((n or 2 ** 14),)
        N = size[0]
        beta = _sparse_beta(rng, N, 0.02)
        keep = gap_mask_1d(rng, N, 0.15, 20)
        lam_factor = 0.1
    elif kind == "2d":
        size = tuple(dims) if dims else ((n or 1024), (n or 1024))
        N = size[0] * size[1]
        beta = _sparse_beta(rng, N, 0.01)
        keep = lattice_mask(size, 32, 4) & (rng.random(N) >= 0.05)
        lam_factor = 0.1
    elif kind == "3d":
        size = tuple(dims) if dims else ((n or 256),) * 3
        N = int(np.prod(size))
        beta = _sparse_beta(rng, N, 0.005, lognormal=True)
        keep = lattice_mask(size, 16, 3)
        lam_factor = 0.05
    else:
        raise ValueError(kind)
    for s in size:
        if s < 2 or s % 2:
            raise ValueError(f"every dimension must be even and >= 2, got {size}")
    noise = 0.01 * rng.standard_normal(N)
    return ProblemSpec(kind, size, beta, keep, noise, lam_factor, seed)


def finalize(spec, synth, apply_At=None):
    """z0 = mask * (A_full beta_true + noise); lambda = lam_factor * ||A^T z0||_inf.

    synth(beta) -> A_full beta (unmasked); apply_At(z) -> A^T z (unmasked).
    """
    x = np.asarray(synth(spec.beta_true), dtype=np.float64)
    y = x + spec.noise
    z0 = np.where(spec.keep, y, 0.0)
    if apply_At is None:
        raise ValueError("apply_At is required to set lambda")
    b = np.asarray(apply_At(z0), dtype=np.float64)
    lam = float(spec.lam_factor * np.abs(b).max())
    missing = np.flatnonzero(~spec.keep).astype(np.int64)
    return Problem(spec, z0, lam, missing)


def known_answer_signal(size):
    """The noiseless separable sinusoids of the reference's end-to-end checks
    (test/ipm_example_1D.jl:6-9, test/ipm_example_2D.jl:7, test/ipm_example_3D.jl:8)."""
    size = tuple(size)
    if len(size) == 1:
        Nt = size[0]
        t = np.arange(Nt, dtype=np.float64)
        return (2 * np.cos(2 * math.pi * t * 6 / Nt) + 3 * np.sin(2 * math.pi * t * 6 / Nt)
                + 4 * np.cos(2 * math.pi * t * 10 / Nt) + 5 * np.sin(2 * math.pi * t * 10 / Nt)
                + 6 * np.cos(2 * math.pi * t * 40 / Nt) + 7 * np.sin(2 * math.pi * t * 40 / Nt))
    if len(size) == 2:
        Nt, Ns = size
        t = np.arange(Nt, dtype=np.float64)
        s = np.arange(Ns, dtype=np.float64)
        a = np.cos(2 * math.pi * 2 / Nt * t) + 2 * np.sin(2 * math.pi * 2 / Nt * t)
        c = np.cos(2 * math.pi * 3 / Ns * s) + 2 * np.sin(2 * math.pi * 3 / Ns * s)
        return np.outer(a, c).ravel(order="F")
    N1, N2, N3 = size
    i = np.arange(N1, dtype=np.float64)
    j = np.arange(N2, dtype=np.float64)
    k = np.arange(N3, dtype=np.float64)
    a = np.cos(2 * math.pi * 1 / N1 * i) + 2 * np.sin(2 * math.pi * 1 / N1 * i)
    b = np.cos(2 * math.pi * 2 / N2 * j) + 2 * np.sin(2 * math.pi * 2 / N2 * j)
    c = np.cos(2 * math.pi * 3 / N3 * k) + 2 * np.sin(2 * math.pi * 3 / N3 * k)
    return np.einsum("i,j,k->ijk", a, b, c).ravel(order="F")


# ------------------------------------------------------------------ serving stream
SERVE_RANGES = {"1d": (2 ** 12, 2 ** 20), "2d": (128, 1024), "3d": (32, 128)}


def smooth_even(rng, lo, hi):
    """A log-uniform draw in [lo, hi] moved to the nearest even number whose
    prime factors are 2, 3 and 5."""
    x = float(np.exp(rng.uniform(np.log(lo), np.log(hi))))
    best = None
    for a in range(1, 21):
        for b in range(0, 13):
            for c in range(0, 9):
                v = (2 ** a) * (3 ** b) * (5 ** c)
                if lo <= v <= hi and (best is None or abs(np.log(v / x)) < abs(np.log(best / x))):
                    best = v
    return best


def serving_spec(seed, max_1d=None):
    """One request of the serving stream: kind uniform over 1D/2D/3D; each
    dimension log-uniform in its range (1D N in [2^12, 2^20], 2D sides in
    [128, 1024], 3D sides in [32, 128]) with factors 2, 3, 5; sparsity
    0.5-5% (N(0,1), log-normal with random signs in 3D); 5-20% missing (gaps
    in 1D, a punched lattice topped up with random samples in 2D/3D);
    sigma = 0.01; lambda factor 0.05-0.1; FP64 or mixed precision.
    ``max_1d`` caps the 1D length."""
    rng = np.random.default_rng(seed)
    kind = ["1d", "2d", "3d"][rng.integers(3)]
    lo, hi = SERVE_RANGES[kind]
    if kind == "1d" and max_1d:
        hi = min(hi, max_1d)
    nd = int(kind[0])
    size = tuple(smooth_even(rng, lo, hi) for _ in range(nd))
    N = int(np.prod(size))
    frac = rng.uniform(0.005, 0.05)
    beta = _sparse_beta(rng, N, frac, lognormal=(kind == "3d"))
    miss = rng.uniform(0.05, 0.20)
    if kind == "1d":
        keep = gap_mask_1d(rng, N, miss, int(rng.integers(5, 30)))
    else:
        keep = lattice_mask(size, 16, 3 if kind == "3d" else 2)
        extra = max(0.0, miss - (1.0 - keep.mean()))
        keep &= rng.random(N) >= extra
    noise = 0.01 * rng.standard_normal(N)
    spec = ProblemSpec(kind, size, beta, keep, noise, float(rng.uniform(0.05, 0.1)), seed)
    precision = "mixed" if rng.random() < 0.5 else "fp64"
    return spec, precision
