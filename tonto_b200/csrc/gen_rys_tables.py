"""Generate the piecewise-polynomial Rys quadrature tables used by the CUDA kernels.

Rys quadrature replaces the Boys-function integral
    F(x)[f] = int_0^1 f(t^2) exp(-x t^2) dt
by an n-point Gauss rule sum_i w_i f(u_i) with nodes u_i = t_i^2 in (0, 1).  Tonto
evaluates the nodes and weights with hand-fitted piecewise polynomials in x
(rys.foo: get_weights and get_weights1_t2 .. get_weights6, :89-3427) and an
asymptotic Gauss-Hermite form for large x.  This script builds tables of the same
kind from first principles:

* exact nodes/weights are computed in 50-digit arithmetic (mpmath) from the Boys
  moments mu_k = F_k(x) = 1F1(k+1/2; k+3/2; -x)/(2k+1), the modified Chebyshev
  (Wheeler) algorithm for the three-term recurrence, and the eigen-decomposition of
  the Jacobi matrix (Golub-Welsch);
* on every unit interval [j, j+1) of x below a cutoff X_n the 2n functions
  u_i(x), w_i(x) are interpolated at DEG+1 Chebyshev points and re-expanded as
  monomials in s = x - j, so that a kernel evaluates each with DEG fused
  multiply-adds (Horner);
* above X_n the asymptotic rule u_i = r_i^2 / x, w_i = W_i / sqrt(x) is used, where
  r_i > 0 are the positive roots of the Hermite polynomial H_{2n} and W_i their
  Gauss-Hermite weights.  X_n is the first even x at which the asymptotic rule
  agrees with the exact one to 1e-17 relative.

The output is a C include file (hex-float literals, so the doubles are exact) plus a
JSON file of reference nodes/weights at random x for the tests.

Usage:  python gen_rys_tables.py [--nmax 9] [--jobs 8]
"""

import argparse
import json
import os
import random
import sys
from multiprocessing import get_context

import mpmath as mp

DEG = 11            # polynomial degree per unit interval
XMAX = {1: 42, 2: 50, 3: 56, 4: 64, 5: 70, 6: 76, 7: 80, 8: 86, 9: 92}
DPS = 50


def boys(m, x):
    x = mp.mpf(x)
    if x == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -x) / (2 * m + 1)


def rys_exact(n, x):
    """Nodes u_i = t_i^2 (ascending) and weights w_i of the n-point Rys rule at x."""
    mp.mp.dps = DPS
    mu = [boys(k, x) for k in range(2 * n)]
    # modified Chebyshev algorithm with ordinary moments
    alpha = [mu[1] / mu[0]]
    beta = [mu[0]]
    s_prev = [mp.mpf(0)] * (2 * n)
    s_cur = list(mu)
    for k in range(1, n):
        s_new = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            s_new[l] = s_cur[l + 1] - alpha[k - 1] * s_cur[l] - beta[k - 1] * s_prev[l]
        alpha.append(s_new[k + 1] / s_new[k] - s_cur[k] / s_cur[k - 1])
        beta.append(s_new[k] / s_cur[k - 1])
        s_prev, s_cur = s_cur, s_new
    J = mp.matrix(n, n)
    for i in range(n):
        J[i, i] = alpha[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(beta[i + 1])
    E, Q = mp.eigsy(J)
    pairs = sorted((E[i], beta[0] * Q[0, i] ** 2) for i in range(n))
    return [p[0] for p in pairs], [p[1] for p in pairs]


def hermite_half(n):
    """Positive roots r_i of H_{2n} (ascending) and their Gauss-Hermite weights."""
    mp.mp.dps = DPS
    import numpy as np
    x, _ = np.polynomial.hermite.hermgauss(2 * n)
    out = []
    for xi in x:
        if xi > 0:
            r = mp.findroot(lambda t: mp.hermite(2 * n, t), mp.mpf(float(xi)))
            W = (mp.mpf(2) ** (2 * n - 1) * mp.factorial(2 * n) * mp.sqrt(mp.pi)) / (
                (2 * n) ** 2 * mp.hermite(2 * n - 1, r) ** 2)
            out.append((r, W))
    out.sort()
    return out


def interval_coefs(args):
    """Monomial coefficients (in s = x - j) for the 2n functions on [j, j+1)."""
    n, j = args
    mp.mp.dps = DPS
    m = DEG + 1
    nodes = [(1 - mp.cos(mp.pi * (k + mp.mpf(1) / 2) / m)) / 2 for k in range(m)]   # in [0,1]
    vals = [rys_exact(n, j + s) for s in nodes]
    funcs = []
    for fi in range(2 * n):
        fv = [(v[0][fi] if fi < n else v[1][fi - n]) for v in vals]
        # solve the Vandermonde system in high precision (well posed at 50 digits)
        V = mp.matrix(m, m)
        for r in range(m):
            for c in range(m):
                V[r, c] = nodes[r] ** c
        a = mp.lu_solve(V, mp.matrix(fv))
        funcs.append([a[c] for c in range(m)])
    return n, j, funcs


def horner(c, s):
    v = 0.0
    for a in reversed(c):
        v = v * s + a
    return v


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nmax", type=int, default=9)
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "rys_tables.inc"))
    ap.add_argument("--golden", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "..",
                                                      "tests", "golden", "rys_reference.json"))
    args = ap.parse_args()
    nmax = args.nmax
    work = [(n, j) for n in range(1, nmax + 1) for j in range(XMAX[n])]
    with get_context("spawn").Pool(args.jobs) as pool:
        res = pool.map(interval_coefs, work, chunksize=4)
    table = {}
    for n, j, funcs in res:
        table[(n, j)] = [[float(a) for a in f] for f in funcs]
    herm = {n: hermite_half(n) for n in range(1, nmax + 1)}

    # accuracy check of the double-precision tables against the exact rule
    rng = random.Random(20241203)
    golden = []
    worst = 0.0
    for n in range(1, nmax + 1):
        xs = [0.0, 1e-12, 1e-6] + [rng.uniform(0, XMAX[n]) for _ in range(40)] + \
             [rng.uniform(XMAX[n], 3 * XMAX[n]) for _ in range(6)]
        for x in xs:
            u, w = rys_exact(n, x)
            if x < XMAX[n]:
                j = int(x)
                s = x - j
                ut = [horner(table[(n, j)][i], s) for i in range(n)]
                wt = [horner(table[(n, j)][n + i], s) for i in range(n)]
            else:
                ut = [float(r) ** 2 / x for r, _ in herm[n]]
                wt = [float(W) / x ** 0.5 for _, W in herm[n]]
            for i in range(n):
                worst = max(worst, abs(ut[i] - float(u[i])) / float(u[i]), abs(wt[i] - float(w[i])) / float(w[i]))
            golden.append({"n": n, "x": x, "u": [mp.nstr(v, 20) for v in u], "w": [mp.nstr(v, 20) for v in w]})
    print("max relative error of tables vs exact:", worst)

    lines = []
    lines.append("// Rys quadrature tables: generated by gen_rys_tables.py (do not edit).")
    lines.append("// Nodes u = t^2 and weights w of the n-point rule for int_0^1 f(t^2) exp(-x t^2) dt.")
    lines.append("// For x < XMAX[n]: on [j, j+1) each function is sum_k coef[k] * (x - j)^k, k = 0..DEG.")
    lines.append("// For x >= XMAX[n]: u_i = hroot2[i] / x and w_i = hweight[i] / sqrt(x).")
    lines.append("// Max relative error against 50-digit Golub-Welsch values: %.2e" % worst)
    lines.append("#define TF_RYS_NMAX %d" % nmax)
    lines.append("#define TF_RYS_DEG %d" % DEG)
    lines.append("#define TF_RYS_NCOEF %d" % (DEG + 1))
    xm = [0] + [XMAX[n] for n in range(1, nmax + 1)]
    lines.append("#define TF_RYS_XMAX_INIT {%s}" % ", ".join(str(v) for v in xm))
    offs = [0]
    tot = 0
    for n in range(1, nmax + 1):
        offs.append(tot)
        tot += XMAX[n] * 2 * n * (DEG + 1)
    lines.append("#define TF_RYS_OFFSET_INIT {%s}" % ", ".join(str(v) for v in offs))
    lines.append("#define TF_RYS_TABLE_SIZE %d" % tot)
    lines.append("TF_RYS_CONST double tf_rys_coef[%d] = {" % tot)
    for n in range(1, nmax + 1):
        for j in range(XMAX[n]):
            row = []
            for f in table[(n, j)]:
                row.extend(float(a).hex() for a in f)
            lines.append("  " + ", ".join(row) + ",  // n=%d j=%d" % (n, j))
    lines.append("};")
    hoff = [0]
    ht = 0
    for n in range(1, nmax + 1):
        hoff.append(ht)
        ht += n
    lines.append("#define TF_RYS_HOFFSET_INIT {%s}" % ", ".join(str(v) for v in hoff))
    r2 = []
    ww = []
    for n in range(1, nmax + 1):
        for r, W in herm[n]:
            r2.append(float(r ** 2).hex())
            ww.append(float(W).hex())
    # the small asymptotic tables may live in a faster memory space than the large one
    lines.append("#ifndef TF_RYS_SMALL_CONST")
    lines.append("#define TF_RYS_SMALL_CONST TF_RYS_CONST")
    lines.append("#endif")
    lines.append("TF_RYS_SMALL_CONST double tf_rys_hroot2[%d] = {%s};" % (ht, ", ".join(r2)))
    lines.append("TF_RYS_SMALL_CONST double tf_rys_hweight[%d] = {%s};" % (ht, ", ".join(ww)))
    with open(args.out, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    with open(args.golden, "w") as fh:
        json.dump({"generator": "tonto_b200/csrc/gen_rys_tables.py", "points": golden}, fh, indent=0)
    print("wrote", args.out, "and", args.golden)


if __name__ == "__main__":
    sys.exit(main())
