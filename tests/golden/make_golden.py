"""Generates tests/golden/known_answers.npz — the reference's own known-answer
cases, computed analytically (no FFT library involved).

The reference's end-to-end checks (test/ipm_example_{1,2,3}D.jl with
check=true) build noiseless separable sinusoids x, take no missing samples and
lambda = 0, and assert that the IPM returns beta_true = DFT_to_beta(fft(x)/sqrt(N))
within 1e-6.  For these signals fft(x) has a handful of nonzero bins that are
known in closed form:  a*cos(2*pi*f*t/n) + b*sin(2*pi*f*t/n) has DFT
n*(a - i b)/2 at bin f and n*(a + i b)/2 at bin n-f, and a separable product
transforms to the outer product of the factors' DFTs.  The spectrum is
assembled from those values and packed with the oracle's restatement of
src/mapping_cpu_kernels.jl (DFT_to_beta), which the map tests pin separately.

Run:  python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "compressedsensingipm.jl_b200"))

import oracle as O                                  # noqa: E402
from csipm.problems import known_answer_signal      # noqa: E402


def dft_1d_terms(n, terms):
    """terms: list of (f, a, b) for a*cos + b*sin at bin f; returns the length-n DFT."""
    v = np.zeros(n, dtype=np.complex128)
    for f, a, b in terms:
        v[f] += n * (a - 1j * b) / 2
        v[(n - f) % n] += n * (a + 1j * b) / 2
    return v


def spectrum(size):
    size = tuple(size)
    if len(size) == 1:
        (n,) = size
        return dft_1d_terms(n, [(6, 2, 3), (10, 4, 5), (40, 6, 7)])
    if len(size) == 2:
        nt, ns = size
        a = dft_1d_terms(nt, [(2, 1, 2)])
        c = dft_1d_terms(ns, [(3, 1, 2)])
        return np.asfortranarray(np.outer(a, c))
    n1, n2, n3 = size
    a = dft_1d_terms(n1, [(1, 1, 2)])
    b = dft_1d_terms(n2, [(2, 1, 2)])
    c = dft_1d_terms(n3, [(3, 1, 2)])
    return np.asfortranarray(np.einsum("i,j,k->ijk", a, b, c))


# the sizes the reference runs its known-answer solves on (test/unit_tests_ipm.jl)
# restricted to those whose test frequencies fit below N/2 (bin 40 needs N > 80 in 1D)
CASES = [(100,), (200,), (500,), (16, 16), (12, 18), (16, 24), (32, 32),
         (8, 8, 8), (6, 10, 12), (14, 8, 4), (8, 6, 4), (16, 16, 16)]


def main():
    out = {}
    for size in CASES:
        N = int(np.prod(size))
        v = spectrum(size) / np.sqrt(N)
        beta = O.dft_to_beta(v, size, impl="kern")
        key = "x".join(str(s) for s in size)
        out[f"x_{key}"] = known_answer_signal(size)
        out[f"beta_{key}"] = beta
    np.savez_compressed(os.path.join(HERE, "known_answers.npz"), **out)
    print("wrote", len(CASES), "cases")


if __name__ == "__main__":
    main()
