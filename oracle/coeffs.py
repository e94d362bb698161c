"""TEST INFRASTRUCTURE -- staggered-grid Taylor coefficients, derived exactly.

For a half-width N the staggered first-derivative weights c_1..c_N solve
    sum_k c_k (2k-1)^(2n-1) = [n == 1],   n = 1..N
(exact rational arithmetic), then are rounded to float32.  For N = 6 the
reference hard-codes eight-digit literals (P-S-seperating.cu:221) whose last
weight differs from the rounded exact value by one float ulp; those literals
are what the reference computes with, so N = 6 uses them.

Run as a script, prints the float32 weights for N (argv[1]) as a C
initialiser body, padded with zeros to six terms: the reference's kernels
unroll exactly six terms (P-S-seperating.cu:224-229), so a half-width below 6
is expressed there by zero weights.
"""
from fractions import Fraction
import sys

import numpy as np

REFERENCE_N6 = (1.2213364, -9.6931458e-2, 1.7447662e-2, -2.9672895e-3, 3.5900540e-4, -2.1847812e-5)
# The reference's first-order velocity/stress kernels (P-S-seperating.cu:405,
# 501) carry five-digit literals of the same weights.
REFERENCE_FO_N6 = (1.2213e+0, -9.6931e-2, 1.7448e-2, -2.9673e-3, 3.5901e-4, -2.1848e-5)


def exact(n):
    rows = [[Fraction((2 * k - 1) ** (2 * p - 1)) for k in range(1, n + 1)] + [Fraction(int(p == 1))]
            for p in range(1, n + 1)]
    for c in range(n):
        piv = next(r for r in range(c, n) if rows[r][c] != 0)
        rows[c], rows[piv] = rows[piv], rows[c]
        for r in range(n):
            if r != c and rows[r][c] != 0:
                f = rows[r][c] / rows[c][c]
                rows[r] = [x - f * y for x, y in zip(rows[r], rows[c])]
    return [rows[i][n] / rows[i][i] for i in range(n)]


def float32_weights(n):
    if n == 6:
        return [np.float32(v) for v in REFERENCE_N6]
    return [np.float32(float(v)) for v in exact(n)]


def float32_weights_first_order(n):
    if n == 6:
        return [np.float32(v) for v in REFERENCE_FO_N6]
    return float32_weights(n)


if __name__ == "__main__":
    n = int(sys.argv[1])
    w = [repr(float(v)) for v in float32_weights(n)] + ["0.0"] * (6 - n)
    print(", ".join(w))
