"""Generate bessel_j01_table.h: piecewise Chebyshev expansions of J_0 and J_1 on the
intervals [a/4, (a+1)/4), a = 0..67, used by the device Bessel code for x < 17.

Coefficients come from Chebyshev interpolation of mpmath values (40 digits) at 48
Chebyshev points per interval, truncated where they fall below 1e-18 (10 per interval; unit
intervals needed 14).

Usage: python nufht_b200/csrc/gen_bessel_table.py   (rewrites the header beside it)
"""
import os

import mpmath as mp

mp.mp.dps = 40
PER_UNIT = 4          # intervals per unit of x
NINT = 17 * PER_UNIT
NODES = 48
CUT = 1e-18


def cheb_coeffs(f, a):
    n = NODES
    th = [mp.pi * (j + mp.mpf(1) / 2) / n for j in range(n)]
    xs = [(a + (mp.cos(t) + 1) / 2) / PER_UNIT for t in th]
    fx = [f(x) for x in xs]
    c = []
    for k in range(n):
        s = mp.fsum(fx[j] * mp.cos(k * th[j]) for j in range(n))
        c.append(2 * s / n)
    c[0] /= 2
    return c


def main():
    rows = {0: [], 1: []}
    deg = 0
    for order in (0, 1):
        for a in range(NINT):
            c = cheb_coeffs(lambda x: mp.besselj(order, x), a)
            d = max(k for k in range(len(c)) if abs(c[k]) > CUT)
            deg = max(deg, d)
            rows[order].append(c)
    ncoef = deg + 1
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "bessel_j01_table.h")
    with open(out, "w") as f:
        f.write("// Generated by gen_bessel_table.py: Chebyshev coefficients of J_0 and J_1 on\n")
        f.write("// [a/%d, (a+1)/%d), a = 0..%d, in t = 2 (%d x - a) - 1.  Do not edit by hand.\n"
                % (PER_UNIT, PER_UNIT, NINT - 1, PER_UNIT))
        f.write("#pragma once\n\nnamespace hankel {\n\n")
        f.write("constexpr int kJ01PerUnit = %d;\nconstexpr int kJ01Intervals = %d;\nconstexpr int kJ01Coefs = %d;\n\n"
                % (PER_UNIT, NINT, ncoef))
        f.write("__device__ const double kJ01Cheb[2][kJ01Intervals][kJ01Coefs] = {\n")
        for order in (0, 1):
            f.write("  {\n")
            for a in range(NINT):
                vals = ", ".join(mp.nstr(rows[order][a][k], 20, strip_zeros=False, min_fixed=0, max_fixed=0)
                                 for k in range(ncoef))
                f.write("    {%s},\n" % vals)
            f.write("  },\n")
        f.write("};\n\n}  // namespace hankel\n")
    print(out, "coefficients per interval:", ncoef)


if __name__ == "__main__":
    main()
