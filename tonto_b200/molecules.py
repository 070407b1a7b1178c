"""Synthetic molecules of the benchmark workloads, and the fixture molecules.

* Water clusters: each water has O-H 0.9572 A and H-O-H 104.52 deg, a seeded random
  orientation, and its O on a 2.8 A simple-cubic lattice with a seeded +-0.2 A
  uniform jitter per coordinate.  Lattice sites are taken from a k x k x k cube
  (k = ceil(n^(1/3))) in (z, y, x) order, so (H2O)_4 fills a 2x2x1 layer and
  (H2O)_32 a 4x4x2 slab.
* Cluster batch: 256 water clusters with n seeded-uniform in [2, 24] (48-576
  cc-pVDZ functions), cluster i built with seed 300000 + i.
* All-trans alkane CnH(2n+2): C-C 1.54 A, C-H 1.09 A, tetrahedral angles, carbon
  zig-zag in the xy plane, seeded +-0.02 A uniform jitter per coordinate.
"""

from __future__ import annotations

import math
from typing import List, Tuple

import numpy as np

from .basis import BOHR_PER_ANGSTROM, Molecule, build_molecule

OH = 0.9572
HOH = math.radians(104.52)
LATTICE = 2.8


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster_geometry(n: int, seed: int) -> Tuple[List[int], np.ndarray]:
    """Z list and coordinates (angstrom) of a seeded (H2O)_n cluster."""
    rng = np.random.default_rng(seed)
    k = max(1, int(math.ceil(n ** (1.0 / 3.0) - 1e-9)))
    sites = [(x, y, z) for z in range(k) for y in range(k) for x in range(k)][:n]
    h1 = np.array([OH * math.sin(HOH / 2), OH * math.cos(HOH / 2), 0.0])
    h2 = np.array([-OH * math.sin(HOH / 2), OH * math.cos(HOH / 2), 0.0])
    Z: List[int] = []
    xyz = []
    for s in sites:
        o = np.array(s, dtype=float) * LATTICE + rng.uniform(-0.2, 0.2, size=3)
        R = _random_rotation(rng)
        Z += [8, 1, 1]
        xyz += [o, o + R @ h1, o + R @ h2]
    return Z, np.array(xyz)


def water_cluster(n: int, seed: int = 0, basis: str = "cc-pVDZ", spherical: bool = True) -> Molecule:
    Z, xyz = water_cluster_geometry(n, seed)
    return build_molecule(Z, xyz * BOHR_PER_ANGSTROM, basis, spherical=spherical)


CLUSTER_BATCH_SIZE_SEED, CLUSTER_BATCH_SEED0 = 3, 300000


def cluster_batch(n_mol: int = 256, lo: int = 2, hi: int = 24, spherical: bool = True) -> List[Molecule]:
    """The batch workload: water clusters with n seeded-uniform in [lo, hi]; the
    first n_mol of the 256-cluster sequence (cluster i has seed 300000 + i)."""
    sizes = np.random.default_rng(CLUSTER_BATCH_SIZE_SEED).integers(lo, hi + 1, size=max(256, n_mol))
    return [water_cluster(int(sizes[i]), seed=CLUSTER_BATCH_SEED0 + i, spherical=spherical) for i in range(n_mol)]


def alkane_geometry(n_c: int, seed: int) -> Tuple[List[int], np.ndarray]:
    """All-trans CnH(2n+2), coordinates in angstrom."""
    rng = np.random.default_rng(seed)
    cc, ch = 1.54, 1.09
    tet = math.acos(-1.0 / 3.0)
    dx = cc * math.sin(tet / 2)
    dy = cc * math.cos(tet / 2)
    C = [np.array([i * dx, (dy / 2) * (1 if i % 2 == 0 else -1), 0.0]) for i in range(n_c)]
    Z: List[int] = [6] * n_c
    xyz = list(C)
    z_axis = np.array([0.0, 0.0, 1.0])

    def virtual(i):   # the zig-zag continuation beyond either chain end
        return np.array([i * dx, (dy / 2) * (1 if i % 2 == 0 else -1), 0.0])

    for i in range(n_c):
        left = C[i - 1] if i > 0 else virtual(-1)
        right = C[i + 1] if i < n_c - 1 else virtual(n_c)
        u1 = (left - C[i]) / np.linalg.norm(left - C[i])
        u2 = (right - C[i]) / np.linalg.norm(right - C[i])
        bis = -(u1 + u2)
        bis /= np.linalg.norm(bis)
        for sgn in (1.0, -1.0):
            d = bis * math.cos(tet / 2) + sgn * z_axis * math.sin(tet / 2)
            Z.append(1)
            xyz.append(C[i] + ch * d)
        if i == 0:
            Z.append(1)
            xyz.append(C[i] + ch * u1)
        if i == n_c - 1:
            Z.append(1)
            xyz.append(C[i] + ch * u2)
    xyz = np.array(xyz) + rng.uniform(-0.02, 0.02, size=(len(xyz), 3))
    return Z, xyz


def alkane(n_c: int = 40, seed: int = 0, basis: str = "def2-SVP", spherical: bool = True) -> Molecule:
    Z, xyz = alkane_geometry(n_c, seed)
    return build_molecule(Z, xyz * BOHR_PER_ANGSTROM, basis, spherical=spherical)


def from_angstrom(Z, xyz_angstrom, basis: str, spherical: bool) -> Molecule:
    return build_molecule(Z, np.asarray(xyz_angstrom, dtype=float) * BOHR_PER_ANGSTROM, basis, spherical=spherical)
