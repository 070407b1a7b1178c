"""The synthetic benchmark inputs follow their specification: water clusters (O-H
0.9572 A, H-O-H 104.52 deg, O on a 2.8 A cubic lattice with +-0.2 A jitter), the
256-cluster batch (2-24 waters, 48-576 cc-pVDZ functions), and all-trans C40H82
(C-C 1.54 A, C-H 1.09 A, +-0.02 A jitter per coordinate, 970 def2-SVP functions)."""

import math

import numpy as np

from tonto_b200.molecules import alkane, alkane_geometry, cluster_batch, water_cluster, water_cluster_geometry


def test_water_clusters():
    for n, seed in ((4, 0), (32, 0), (13, 7)):
        Z, xyz = water_cluster_geometry(n, seed)
        assert Z == [8, 1, 1] * n
        k = math.ceil(n ** (1.0 / 3.0) - 1e-9)
        sites = [(x, y, z) for z in range(k) for y in range(k) for x in range(k)][:n]
        for w in range(n):
            o, h1, h2 = xyz[3 * w:3 * w + 3]
            assert abs(np.linalg.norm(h1 - o) - 0.9572) < 1e-12 and abs(np.linalg.norm(h2 - o) - 0.9572) < 1e-12
            cosang = np.dot(h1 - o, h2 - o) / 0.9572 ** 2
            assert abs(math.degrees(math.acos(cosang)) - 104.52) < 1e-9
            assert np.max(np.abs(o - 2.8 * np.array(sites[w], dtype=float))) <= 0.2
    assert water_cluster(4).n_bf == 96 and water_cluster(32).n_bf == 768


def test_cluster_batch():
    a = cluster_batch(256)
    b = cluster_batch(256)
    sizes = [m.n_atom // 3 for m in a]
    assert min(sizes) >= 2 and max(sizes) <= 24 and len(set(sizes)) > 10
    assert all(48 <= m.n_bf <= 576 for m in a)
    assert all(np.array_equal(x.xyz, y.xyz) for x, y in zip(a, b))   # seeded
    assert [m.n_bf for m in cluster_batch(64)] == [m.n_bf for m in a[:64]]


def test_alkane():
    Z, xyz = alkane_geometry(40, 0)
    assert Z.count(6) == 40 and Z.count(1) == 82
    C = xyz[:40]
    jit = 2 * math.sqrt(3) * 0.02                     # two atoms, +-0.02 A per coordinate
    cc = np.linalg.norm(C[1:] - C[:-1], axis=1)
    assert np.all(np.abs(cc - 1.54) <= jit)
    H = xyz[40:]
    ch = np.min(np.linalg.norm(H[:, None, :] - C[None, :, :], axis=2), axis=1)
    assert np.all(np.abs(ch - 1.09) <= jit)
    assert alkane(40).n_bf == 970
