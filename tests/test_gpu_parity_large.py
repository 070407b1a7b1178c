"""Per-element parity at the measured workloads: the FP64 J and K of (H2O)32 cc-pVDZ
(768 spherical functions) and of all-trans C40H82 def2-SVP (970 spherical
functions), Schwarz cutoff 1e-12, from the core-Hamiltonian guess density, against
the oracle's restatement of make_r_JK_direct (molecule.fock.foo:1235-1363), to
1e-11 max-abs per element; and the screening: the library's per-class counts of
contracted and primitive quartets equal the oracle's to the unit
(Schwarz_inequality_test :3454-3495 and the primitive-pair cutoff,
shell1quartet.foo:229-273).  The oracle runs on all host cores (about 20 s each)."""

import numpy as np
import pytest

TOL = 1e-11


def _core_density(oracle_mod, orc, mol):
    S, T, V = orc.one_electron()
    P, _, _ = oracle_mod.density_from_fock(T + V, oracle_mod.orthogonaliser(S), mol.n_electrons // 2)
    return P


def _check_workload(oracle_mod, mol):
    from tonto_b200.fock import FockBuilder
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P = _core_density(oracle_mod, orc, mol)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    fb.set_graph(False)                        # class-by-class build: per-class counts of this build
    J, K = fb.make_r_JK(P)
    cls = {c["class"]: c for c in fb.class_stats()}
    fb.set_graph(True)
    Jg, Kg = fb.make_r_JK(P)                   # and the captured-graph build
    fb.close()
    orc.counts(reset=True)
    Jr, Kr = orc.jk(P)
    cnt = orc.counts(reset=True).reshape(625, 2)
    dJ, dK = float(np.max(np.abs(J - Jr))), float(np.max(np.abs(K - Kr)))
    assert dJ <= TOL and dK <= TOL, (dJ, dK)
    assert float(np.max(np.abs(Jg - Jr))) <= TOL and float(np.max(np.abs(Kg - Kr))) <= TOL
    sym = "spdfg"
    ref = {}
    for q in range(625):
        if cnt[q, 0] > 0:
            l = (q // 125, (q // 25) % 5, (q // 5) % 5, q % 5)
            ref["(%s%s|%s%s)" % tuple(sym[v] for v in l)] = (cnt[q, 0], cnt[q, 1])
    got = {k: (v["quartets"], v["prim_quartets"]) for k, v in cls.items() if v["quartets"] > 0}
    assert got == ref
    return dJ, dK


@pytest.mark.gpu
def test_water32_jk_matches_oracle_per_element(cuda_ok, oracle_mod):
    from tonto_b200.molecules import water_cluster
    mol = water_cluster(32, seed=0)
    assert mol.n_bf == 768
    _check_workload(oracle_mod, mol)


@pytest.mark.gpu
def test_alkane_c40_jk_matches_oracle_per_element(cuda_ok, oracle_mod):
    from tonto_b200.molecules import alkane
    mol = alkane(40, seed=0)
    assert mol.n_bf == 970
    _check_workload(oracle_mod, mol)
