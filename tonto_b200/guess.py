"""Initial densities for water clusters: local frames, AO rotations, and the
monomer-superposition guess.

Every water gets a right-handed local frame (origin at O, x along the H-O-H
bisector, y along H1 - H2 within the molecular plane, z = x cross y).  A
density block expressed in local frames is taken to the lab frame with the AO
rotation matrices of the two waters:

    P_lab(v, w) = A_v^T  P_local(v, w)  A_w,

where A is block-diagonal over shells: 1 for s, the 3x3 frame rotation for p
(Tonto's x, y, z order), and for d the 5x5 (spherical) or 6x6 (Cartesian)
representation of the same rotation on Tonto's solid harmonics / Cartesian
components.  The monomer-superposition guess places the converged isolated
water density (in its local frame) on every water — the analogue of Tonto's
promolecule guess (molecule.scf.foo:4827) for a cluster of identical molecules.
"""

from __future__ import annotations

import itertools
import math
from functools import lru_cache
from typing import List, Tuple

import numpy as np

from .basis import Molecule


# ---------------------------------------------------------------------------
# Cartesian components (Tonto order) and solid-harmonic matrices on the host
# ---------------------------------------------------------------------------
@lru_cache(maxsize=None)
def cart_components(l: int) -> Tuple[Tuple[int, int, int], ...]:
    """Tonto's lexical order (gaussian_data.foo:295-479)."""
    out = []
    L = l
    for a in range(L, (L + 2) // 3 - 1, -1):
        for b in range(min(L - a, a), (L - a + 1) // 2 - 1, -1):
            c = L - a - b
            if a == b == c:
                out.append((a, a, a))
            elif a > b and b == c:
                out += [(a, b, b), (b, a, b), (b, b, a)]
            elif a == b and b > c:
                out += [(a, a, c), (a, c, a), (c, a, a)]
            else:
                out += [(a, b, c), (a, c, b), (b, a, c), (c, a, b), (b, c, a), (c, b, a)]
    return tuple(out)


@lru_cache(maxsize=None)
def solid_harmonics(l: int) -> np.ndarray:
    """ncart(l) x (2l+1) matrix, columns m = 0, +1, -1, +2, -2, ... (Helgaker,
    Jorgensen & Olsen eqs. 6.4.70-73, the recurrence Tonto uses)."""
    def col(m):
        return 0 if m == 0 else (2 * m - 1 if m > 0 else -2 * m)
    S = {0: {(0, 0, 0): {0: 1.0}}}     # S[L][monomial] -> {m: coef}
    for L in range(l):
        nxt = {}
        fac = math.sqrt((2.0 if L == 0 else 1.0) * (2 * L + 1) / (2 * L + 2))
        dl = 0.0 if L == 0 else 1.0

        def add(mono, m, v):
            nxt.setdefault(mono, {})
            nxt[mono][m] = nxt[mono].get(m, 0.0) + v
        for mono, cs in S[L].items():
            x, y, z = mono
            sLL = cs.get(L, 0.0)
            sLm = cs.get(-L, 0.0)
            add((x + 1, y, z), L + 1, fac * sLL)
            add((x, y + 1, z), L + 1, -fac * sLm * dl)
            add((x + 1, y, z), -L - 1, fac * sLm * dl)
            add((x, y + 1, z), -L - 1, fac * sLL)
            for M in range(-L, L + 1):
                if M in cs:
                    add((x, y, z + 1), M, (2 * L + 1) / math.sqrt((L + M + 1) * (L - M + 1)) * cs[M])
        if L >= 1:
            for mono, cs in S[L - 1].items():
                x, y, z = mono
                for M in range(-L + 1, L):
                    if M in cs:
                        v = math.sqrt((L + M) * (L - M) / ((L + M + 1) * (L - M + 1))) * cs[M]
                        add((x + 2, y, z), M, -v)
                        add((x, y + 2, z), M, -v)
                        add((x, y, z + 2), M, -v)
        S[L + 1] = nxt
    comps = cart_components(l)
    U = np.zeros((len(comps), 2 * l + 1))
    for i, c in enumerate(comps):
        for m, v in S[l].get(c, {}).items():
            U[i, col(m)] = v
    return U


def cart_rotation(l: int, R: np.ndarray) -> np.ndarray:
    """C[c, c'] with m_c(R r) = sum_c' C[c, c'] m_c'(r) for the degree-l monomials:
    the product of a copies of row 0, b of row 1 and c of row 2 of R, expanded (the
    outer product of those rows, summed into the monomials its index tuples give)."""
    comps = cart_components(l)
    if l == 0:
        return np.ones((1, 1))
    idx = {c: i for i, c in enumerate(comps)}
    tgt = np.array([idx[tuple(kk.count(d) for d in range(3))] for kk in itertools.product(range(3), repeat=l)])
    C = np.zeros((len(comps), len(comps)))
    for i, (a, b, c) in enumerate(comps):
        rows = [0] * a + [1] * b + [2] * c
        T = R[rows[0]]
        for r in rows[1:]:
            T = np.multiply.outer(T, R[r])
        C[i] = np.bincount(tgt, weights=T.ravel(), minlength=len(comps))
    return C


def shell_rotation(l: int, R: np.ndarray, spherical: bool) -> np.ndarray:
    """A with chi_local = A chi_lab for one shell (R: lab -> local frame rows)."""
    if l == 0:
        return np.ones((1, 1))
    C = cart_rotation(l, R)
    if not spherical or l < 2:
        return C
    U = solid_harmonics(l)
    V = U.T @ C
    return V @ U @ np.linalg.inv(U.T @ U)


# ---------------------------------------------------------------------------
# waters and frames
# ---------------------------------------------------------------------------
def waters(mol: Molecule) -> List[Tuple[int, int, int]]:
    """(O, H1, H2) atom indices, for molecules listed as consecutive O, H, H."""
    Z = list(mol.Z)
    out = []
    i = 0
    while i < len(Z):
        if Z[i] == 8 and i + 2 < len(Z) and Z[i + 1] == 1 and Z[i + 2] == 1:
            out.append((i, i + 1, i + 2))
            i += 3
        else:
            raise ValueError("not a water cluster (atoms must be O, H, H per molecule)")
    return out


def water_frame(xyz: np.ndarray, o: int, h1: int, h2: int) -> np.ndarray:
    """Rows: local x, y, z axes in lab coordinates."""
    O = xyz[o]
    a = xyz[h1] - O
    b = xyz[h2] - O
    x = a + b
    x /= np.linalg.norm(x)
    y = a - b
    y -= x * np.dot(x, y)
    y /= np.linalg.norm(y)
    z = np.cross(x, y)
    return np.stack([x, y, z])


def water_ao_ranges(mol: Molecule) -> List[Tuple[int, int]]:
    """[first, last+1) basis-function range of each water (its atoms' shells)."""
    ranges = []
    for (o, h1, h2) in waters(mol):
        sh = [s for s in mol.shells if s.atom in (o, h1, h2)]
        f0 = sh[0].first_bf
        f1 = sh[-1].first_bf + mol.shell_nbf(sh[-1].l)
        ranges.append((f0, f1))
    return ranges


def water_ao_rotation(mol: Molecule, w: Tuple[int, int, int], R: np.ndarray) -> np.ndarray:
    by_l = {}                                       # one rotation block per angular momentum
    blocks = [by_l.setdefault(s.l, shell_rotation(s.l, R, mol.spherical)) if s.l not in by_l else by_l[s.l]
              for s in mol.shells if s.atom in w]
    n = sum(b.shape[0] for b in blocks)
    A = np.zeros((n, n))
    k = 0
    for b in blocks:
        m = b.shape[0]
        A[k:k + m, k:k + m] = b
        k += m
    return A


def cluster_rotations(mol: Molecule):
    ws = waters(mol)
    frames = [water_frame(mol.xyz, *w) for w in ws]
    A = [water_ao_rotation(mol, w, R) for w, R in zip(ws, frames)]
    return ws, frames, A


def superposition_guess(mol: Molecule, P_mono_local: np.ndarray) -> np.ndarray:
    """Block-diagonal density: the isolated-water density on every water."""
    ws, frames, A = cluster_rotations(mol)
    rng = water_ao_ranges(mol)
    P = np.zeros((mol.n_bf, mol.n_bf))
    for (f0, f1), Aw in zip(rng, A):
        P[f0:f1, f0:f1] = Aw.T @ P_mono_local @ Aw
    return P


def reference_water(basis: str = "cc-pVDZ", spherical: bool = True) -> Molecule:
    """The isolated water in its own local frame (O at the origin)."""
    from .molecules import HOH, OH, from_angstrom
    h1 = [OH * math.cos(HOH / 2), OH * math.sin(HOH / 2), 0.0]
    h2 = [OH * math.cos(HOH / 2), -OH * math.sin(HOH / 2), 0.0]
    return from_angstrom([8, 1, 1], [[0.0, 0.0, 0.0], h1, h2], basis, spherical)


def to_local(P_lab_block: np.ndarray, Av: np.ndarray, Aw: np.ndarray) -> np.ndarray:
    """Inverse of P_lab = Av^T P_local Aw (general; Av, Aw orthogonal in a spherical basis)."""
    return np.linalg.solve(Av.T, np.linalg.solve(Aw.T, P_lab_block.T).T)
