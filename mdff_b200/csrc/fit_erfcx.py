"""Coefficients of erfc_ex2's table c_erfcx (common.cuh).

erfcx(x) = erfc(x) e^{x^2} on each interval [j/2, j/2 + 1/2), j = 0..8, as the
degree-13 polynomial in t = 4x - (2j + 1) in [-1, 1) that interpolates it at
the 14 Chebyshev points t_k = cos((2k + 1) pi / 28), computed in 50-digit
arithmetic (mpmath) and written as monomial coefficients in t, lowest power
first, for Horner evaluation in FP64.

  python mdff_b200/csrc/fit_erfcx.py          # prints the C table
  python mdff_b200/csrc/fit_erfcx.py --check  # compares with common.cuh
"""
import os
import re
import sys

import mpmath as mp

DEG = 13
NINT = 9


def fit(j):
    mp.mp.dps = 50
    nodes = [mp.cos((2 * k + 1) * mp.pi / (2 * (DEG + 1))) for k in range(DEG + 1)]
    f = [mp.erfc((t + 2 * j + 1) / 4) * mp.exp(((t + 2 * j + 1) / 4) ** 2) for t in nodes]
    V = mp.matrix([[t ** p for p in range(DEG + 1)] for t in nodes])
    return mp.lu_solve(V, mp.matrix(f))


def table():
    return [[float(c) for c in fit(j)] for j in range(NINT)]


def committed():
    src = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "common.cuh")).read()
    body = src[src.index("c_erfcx[9][14]"):]
    body = body[body.index("{") + 1:body.index("};")]
    rows = re.findall(r"\{([^{}]*)\}", body)
    return [[float(x) for x in r.split(",")] for r in rows]


if __name__ == "__main__":
    tab = table()
    if "--check" in sys.argv:
        ref = committed()
        worst = max(abs(a - b) / abs(b) for ra, rb in zip(tab, ref) for a, b in zip(ra, rb))
        print("largest relative difference from common.cuh: %.3g" % worst)
        sys.exit(0 if worst < 1e-12 else 1)
    print("static __device__ const double c_erfcx[%d][%d] = {" % (NINT, DEG + 1))
    print(",\n".join("    {" + ", ".join("%.17e" % c for c in row) + "}" for row in tab) + "};")
