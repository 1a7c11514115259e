"""Writes the root-of-unity tables of roots.h for the register DFT sizes
given on the command line: W_R^m = exp(-2*pi*i*m/R), m < R, evaluated in
80-digit decimal arithmetic and rounded once to double (Python's
float(Decimal) rounds correctly).  Angles that are whole multiples of pi/2
give exact 0 and +-1.

    python gen_roots.py 18 24 27 30 > tables.txt
"""
import sys
from decimal import Decimal, getcontext

getcontext().prec = 80


def dec_pi():
    # Machin: pi = 16 atan(1/5) - 4 atan(1/239)
    def atan_inv(n):
        x = Decimal(1) / n
        x2 = x * x
        term, total, k = x, x, 1
        eps = Decimal(10) ** -(getcontext().prec + 2)
        while abs(term) > eps:
            term *= -x2
            total += term / (2 * k + 1)
            k += 1
        return total
    return 16 * atan_inv(5) - 4 * atan_inv(239)


def dec_cos_sin(x):
    # Taylor series; |x| <= pi here, enough terms for 80 digits
    eps = Decimal(10) ** -(getcontext().prec + 2)
    c, s = Decimal(0), Decimal(0)
    term, k = Decimal(1), 0        # x^k / k!
    while True:
        if k % 4 == 0:
            c += term
        elif k % 4 == 1:
            s += term
        elif k % 4 == 2:
            c -= term
        else:
            s -= term
        k += 1
        term = term * x / k
        if abs(term) < eps and k > 4:
            break
    return c, s


def root(m, R, pi):
    """(re, im) of exp(-2 pi i m / R) as doubles."""
    if (4 * m) % R == 0:
        q = (4 * m) // R % 4      # angle = q * pi/2
        return [(1.0, -0.0), (0.0, -1.0), (-1.0, 0.0), (0.0, 1.0)][q]
    # reduce to |angle| <= pi: exp(-2 pi i m/R) = conj(exp(-2 pi i (R-m)/R))
    flip = 2 * m > R
    mm = R - m if flip else m
    c, s = dec_cos_sin(2 * pi * mm / R)
    re, im = float(c), float(-s)
    return (re, -im) if flip else (re, im)


def emit(R, pi):
    vals = [root(m, R, pi) for m in range(R)]
    out = []
    for part, idx in (("re", 0), ("im", 1)):
        out.append(f"__device__ __forceinline__ constexpr double root_{part}{R}(int m) {{")
        out.append("    switch (m) {")
        for m, v in enumerate(vals):
            out.append(f"        case {m}: return {repr(v[idx])};")
        out.append("        default: return 0.0;")
        out.append("    }")
        out.append("}")
    return "\n".join(out)


if __name__ == "__main__":
    pi = dec_pi()
    print("\n".join(emit(int(r), pi) for r in sys.argv[1:]))
