"""Host-side parts of the initial-density guess (no GPU): the pair list and the
environment descriptors against a plain per-pair restatement of their definition, and
the Cartesian rotation blocks against the expansion of the rotated monomials."""

import math

import numpy as np

from tonto_b200 import guess as G
from tonto_b200 import learned_guess as LG
from tonto_b200.molecules import cluster_batch, water_cluster


def _pairs_loop(atoms):
    n = len(atoms)
    out = [(v, v) for v in range(n)]
    for v in range(n):
        for w in range(v + 1, n):
            if np.linalg.norm(atoms[w, 0] - atoms[v, 0]) < LG.PAIR_CUTOFF:
                out.append((v, w))
    return out


def _descriptors_loop(atoms, frames, pairs, env_k):
    fc = lambda r: 0.5 * (math.cos(math.pi * r / LG.RC) + 1.0) if r < LG.RC else 0.0  # noqa: E731
    n = len(atoms)
    X = np.zeros((len(pairs), LG.d_in(env_k)))
    for k, (v, w) in enumerate(pairs):
        R, Ov, f = frames[v], atoms[v, 0], X[k]
        if v == w:
            f[0] = 1.0
            centre = Ov
        else:
            f[1:10] = ((atoms[w] - Ov) @ R.T).ravel()
            f[10] = fc(float(np.linalg.norm(atoms[w, 0] - Ov)))
            centre = 0.5 * (Ov + atoms[w, 0])
        others = sorted((u for u in range(n) if u != v and u != w),
                        key=lambda u: float(np.linalg.norm(atoms[u, 0] - centre)))
        for j, u in enumerate(others[:env_k]):
            f[11 + 10 * j:20 + 10 * j] = ((atoms[u] - Ov) @ R.T).ravel()
            f[20 + 10 * j] = fc(float(np.linalg.norm(atoms[u, 0] - centre)))
    return X


def test_pairs_and_descriptors_match_their_definition():
    mols = cluster_batch(12) + [water_cluster(1, seed=3), water_cluster(2, seed=4), water_cluster(32, seed=0)]
    for m in mols:
        _, frames, _, atoms = LG.cluster_geometry(m)
        pairs = LG.pair_list(atoms)
        assert pairs == _pairs_loop(atoms)
        for env_k in (LG.ENV_K, 8):
            X = LG.descriptors(atoms, frames, pairs, env_k)
            assert np.max(np.abs(X - _descriptors_loop(atoms, frames, pairs, env_k))) < 1e-13


def test_cartesian_rotation_rotates_the_monomials():
    rng = np.random.default_rng(5)
    R = np.linalg.qr(rng.normal(size=(3, 3)))[0]
    r = rng.normal(size=3)
    for l in range(4):
        comps = G.cart_components(l)
        C = G.cart_rotation(l, R)
        mono = lambda x: np.array([x[0] ** a * x[1] ** b * x[2] ** c for a, b, c in comps])  # noqa: E731
        assert np.max(np.abs(mono(R @ r) - C @ mono(r))) < 1e-12
