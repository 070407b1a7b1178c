"""Generate the Boys-function grid used for the one-point Rys rule.

With one root the Rys rule of int_0^1 f(t^2) exp(-x t^2) dt is exact for f linear
in t^2, so its node and weight follow from two Boys functions:
    w = F_0(x),   u = t^2 = F_1(x) / F_0(x).
The kernels evaluate F_0 and F_1 by a Taylor expansion about the nearest point
x_k = k / 8 of a grid on [0, XMAX):
    F_m(x) = sum_{j=0..7} F_{m+j}(x_k) (x_k - x)^j / j!,   |x - x_k| <= 1/16,
using dF_m/dx = -F_{m+1}.  The truncation term is bounded by F_{m+8} (1/16)^8 / 8!,
below 5.8e-15 relative (F_{m+8} <= F_m).  The table holds F_0 .. F_8 at every grid
point, padded to 10 doubles (five 16-byte loads per evaluation, 27 KB in all).  For
x >= XMAX the asymptotic one-point rule of the Rys tables applies (u = 1 / (2x),
w = sqrt(pi / x) / 2).

Boys functions are computed in 50-digit arithmetic (mpmath) as
F_m(x) = 1F1(m + 1/2; m + 3/2; -x) / (2m + 1).

A second grid (boys2_table.inc: F_0 .. F_10 on [0, 50), padded to 12 doubles, 38 KB)
serves the two-point rule, built from the moments F_0..F_3: u_1, u_2 are the roots of
u^2 + a u + b, the monic polynomial orthogonal to 1 and u,
    a = (F0 F3 - F1 F2) / (F1^2 - F0 F2),   b = (F2^2 - F1 F3) / (F1^2 - F0 F2),
taken as q = (sqrt(a^2 - 4b) - a) / 2 (a < 0: no cancellation), u_1 = q, u_2 = b / q;
w_1 = (F0 u_2 - F1) / (u_2 - u_1), w_2 = F0 - w_1.  Its error against 50-digit
Golub-Welsch values is reported too.

Usage:  python gen_boys_table.py
"""

import argparse
import math
import os
import random

import mpmath as mp

from gen_rys_tables import rys_exact

XMAX = 42           # the one-root Rys tables switch to the asymptotic rule here
H_INV = 8           # grid spacing 1/8
NM = 10             # F_0 .. F_8 per grid point, and one pad
NTERM = 8
DPS = 50


def boys(m, x):
    x = mp.mpf(x)
    if x == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -x) / (2 * m + 1)


def taylor(tab, x):
    """F_0, F_1 at x from the double-precision grid, as the kernels compute them."""
    k = int(x * H_INV + 0.5)
    d = k / H_INV - x
    f = tab[k]
    out = []
    for m in (0, 1):
        v = f[m + NTERM - 1]
        for j in range(NTERM - 1, 0, -1):
            v = f[m + j - 1] + (d / j) * v
        out.append(v)
    return out


def taylor_m(tab, x, m, h_inv):
    k = int(x * h_inv + 0.5)
    d = k / h_inv - x
    f = tab[k]
    v = f[m + NTERM - 1]
    for j in range(NTERM - 1, 0, -1):
        v = f[m + j - 1] + (d / j) * v
    return v


def rule2(tab, x):
    m0, m1, m2, m3 = (taylor_m(tab, x, m, H_INV) for m in range(4))
    r = 1.0 / (m1 * m1 - m0 * m2)
    a = (m0 * m3 - m1 * m2) * r
    b = (m2 * m2 - m1 * m3) * r
    q = 0.5 * (math.sqrt(a * a - 4.0 * b) - a)
    u1, u2 = q, b / q
    w1 = (m0 * u2 - m1) / (u2 - u1)
    return sorted([(u1, w1), (u2, m0 - w1)])


def write_two_point(path):
    xmax, nm = 50, 12
    npts = xmax * H_INV + 1
    tab = [[float(boys(m, mp.mpf(k) / H_INV)) for m in range(NTERM + 3)] + [0.0] for k in range(npts)]
    rng = random.Random(20261204)
    worst = 0.0
    for x in [0.0, 1e-12, 1e-3, 0.03125, xmax - 1e-9] + [rng.uniform(0, xmax) for _ in range(3000)]:
        ue, we = rys_exact(2, x)
        for (u, w), uei, wei in zip(rule2(tab, x), ue, we):
            worst = max(worst, abs(u - float(uei)) / float(uei), abs(w - float(wei)) / float(wei))
    print("max relative error of the two-point rule vs exact:", worst)
    lines = ["// Boys-function grid for the two-point Rys rule: generated by gen_boys_table.py (do not edit).",
             "// tf_boys2_grid[k][m] = F_m(k / %d), m = 0..%d (then zero pad), k = 0..%d." % (H_INV, NTERM + 2, npts - 1),
             "// Max relative error of (u, w) against 50-digit values: %.2e" % worst,
             "#define TF_BOYS2_XMAX %d" % xmax,
             "#define TF_BOYS2_NM %d" % nm,
             "#define TF_BOYS2_NPTS %d" % npts,
             "TF_RYS_CONST double tf_boys2_grid[%d] = {" % (npts * nm)]
    for k in range(npts):
        lines.append("  " + ", ".join(v.hex() for v in tab[k]) + ",")
    lines.append("};")
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "boys_table.inc"))
    args = ap.parse_args()
    mp.mp.dps = DPS
    npts = XMAX * H_INV + 1
    tab = [[float(boys(m, mp.mpf(k) / H_INV)) for m in range(NTERM + 1)] + [0.0] * (NM - NTERM - 1)
           for k in range(npts)]
    rng = random.Random(20261203)
    worst = 0.0
    for x in [0.0, 1e-12, 1e-3, 0.03125, XMAX - 1e-9] + [rng.uniform(0, XMAX) for _ in range(4000)]:
        f0, f1 = taylor(tab, x)
        e0, e1 = boys(0, x), boys(1, x)
        u, w = f1 / f0, f0
        worst = max(worst, abs(w - float(e0)) / float(e0), abs(u - float(e1 / e0)) / float(e1 / e0))
    print("max relative error of the one-point rule vs exact:", worst)
    lines = ["// Boys-function grid for the one-point Rys rule: generated by gen_boys_table.py (do not edit).",
             "// tf_boys_grid[k][m] = F_m(k / %d), m = 0..%d (then zero pad), k = 0..%d." % (H_INV, NTERM, npts - 1),
             "// Max relative error of (u, w) from a %d-term Taylor step against 50-digit values: %.2e"
             % (NTERM, worst),
             "#define TF_BOYS_XMAX %d" % XMAX,
             "#define TF_BOYS_H_INV %d" % H_INV,
             "#define TF_BOYS_NM %d" % NM,
             "#define TF_BOYS_NTERM %d" % NTERM,
             "#define TF_BOYS_NPTS %d" % npts,
             "TF_RYS_CONST double tf_boys_grid[%d] = {" % (npts * NM)]
    for k in range(npts):
        lines.append("  " + ", ".join(v.hex() for v in tab[k]) + ",")
    lines.append("};")
    with open(args.out, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    write_two_point(os.path.join(os.path.dirname(args.out), "boys2_table.inc"))


if __name__ == "__main__":
    main()
