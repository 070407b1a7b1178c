"""Independent reference ERIs for tests: McMurchie-Davidson over Hermite Gaussians
with the Boys function from mpmath (1F1), for small contracted Cartesian shells.

Used only to check the oracle's Rys-quadrature integrals on a few quartets; it
shares no code with the oracle or the CUDA library.
"""

import math

import mpmath as mp
import numpy as np


def boys(n, T):
    if T < 1e-15:
        return 1.0 / (2 * n + 1)
    return float(mp.hyp1f1(n + 0.5, n + 1.5, -T) / (2 * n + 1))


def hermite_E(i, j, t, Qx, a, b):
    p = a + b
    q = a * b / p
    if t < 0 or t > i + j:
        return 0.0
    if i == j == t == 0:
        return math.exp(-q * Qx * Qx)
    if j == 0:
        return (1 / (2 * p)) * hermite_E(i - 1, j, t - 1, Qx, a, b) - (q * Qx / a) * hermite_E(i - 1, j, t, Qx, a, b) \
            + (t + 1) * hermite_E(i - 1, j, t + 1, Qx, a, b)
    return (1 / (2 * p)) * hermite_E(i, j - 1, t - 1, Qx, a, b) + (q * Qx / b) * hermite_E(i, j - 1, t, Qx, a, b) \
        + (t + 1) * hermite_E(i, j - 1, t + 1, Qx, a, b)


def hermite_R(t, u, v, n, p, PCx, PCy, PCz, RPC, cache):
    key = (t, u, v, n)
    if key in cache:
        return cache[key]
    T = p * RPC * RPC
    if t == u == v == 0:
        val = (-2 * p) ** n * boys(n, T)
    elif t == u == 0:
        val = (v - 1) * hermite_R(t, u, v - 2, n + 1, p, PCx, PCy, PCz, RPC, cache) if v > 1 else 0.0
        val += PCz * hermite_R(t, u, v - 1, n + 1, p, PCx, PCy, PCz, RPC, cache)
    elif t == 0:
        val = (u - 1) * hermite_R(t, u - 2, v, n + 1, p, PCx, PCy, PCz, RPC, cache) if u > 1 else 0.0
        val += PCy * hermite_R(t, u - 1, v, n + 1, p, PCx, PCy, PCz, RPC, cache)
    else:
        val = (t - 1) * hermite_R(t - 2, u, v, n + 1, p, PCx, PCy, PCz, RPC, cache) if t > 1 else 0.0
        val += PCx * hermite_R(t - 1, u, v, n + 1, p, PCx, PCy, PCz, RPC, cache)
    cache[key] = val
    return val


def prim_eri(a, lmn1, A, b, lmn2, B, c, lmn3, C, d, lmn4, D):
    l1, m1, n1 = lmn1
    l2, m2, n2 = lmn2
    l3, m3, n3 = lmn3
    l4, m4, n4 = lmn4
    p = a + b
    q = c + d
    alpha = p * q / (p + q)
    P = (a * A + b * B) / p
    Q = (c * C + d * D) / q
    RPQ = np.linalg.norm(P - Q)
    cache = {}
    val = 0.0
    for t in range(l1 + l2 + 1):
        Et = hermite_E(l1, l2, t, A[0] - B[0], a, b)
        for u in range(m1 + m2 + 1):
            Eu = hermite_E(m1, m2, u, A[1] - B[1], a, b)
            for v in range(n1 + n2 + 1):
                Ev = hermite_E(n1, n2, v, A[2] - B[2], a, b)
                for tau in range(l3 + l4 + 1):
                    Ft = hermite_E(l3, l4, tau, C[0] - D[0], c, d)
                    for nu in range(m3 + m4 + 1):
                        Fu = hermite_E(m3, m4, nu, C[1] - D[1], c, d)
                        for phi in range(n3 + n4 + 1):
                            Fv = hermite_E(n3, n4, phi, C[2] - D[2], c, d)
                            val += Et * Eu * Ev * Ft * Fu * Fv * (-1) ** (tau + nu + phi) * hermite_R(
                                t + tau, u + nu, v + phi, 0, alpha, P[0] - Q[0], P[1] - Q[1], P[2] - Q[2], RPQ, cache)
    return val * 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q))


def contracted_eri(shells, comps):
    """shells: 4 tuples (exps, coefs, centre); comps: 4 (lx,ly,lz) tuples."""
    (ea, ca, A), (eb, cb, B), (ec, cc, C), (ed, cd, D) = shells
    s = 0.0
    for a, x1 in zip(ea, ca):
        for b, x2 in zip(eb, cb):
            for c, x3 in zip(ec, cc):
                for d, x4 in zip(ed, cd):
                    s += x1 * x2 * x3 * x4 * prim_eri(a, comps[0], A, b, comps[1], B, c, comps[2], C, d, comps[3], D)
    return s
