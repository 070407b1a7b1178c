"""GPU SCF, one-electron integrals and sharded builds against the oracle."""

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster


@pytest.mark.gpu
def test_one_electron_matches_oracle(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    for spherical in (True, False):
        mol = water_cluster(2, seed=3, spherical=spherical)
        orc = oracle_mod.Oracle(mol)
        S0, T0, V0 = orc.one_electron()
        S, T, V = FockBuilder(mol).one_electron()
        for a, b in ((S, S0), (T, T0), (V, V0)):
            assert np.max(np.abs(a - b)) < 1e-11


@pytest.mark.gpu
def test_shards_sum_to_full_build(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(3, seed=9)
    rng = np.random.default_rng(1)
    A = rng.normal(size=(mol.n_bf, mol.n_bf)) * 0.05
    P = A + A.T
    full = FockBuilder(mol, schwarz_cutoff=1e-12)
    J, K = full.make_r_JK(P)
    Js = np.zeros_like(J)
    Ks = np.zeros_like(K)
    for r in range(3):
        fb = FockBuilder(mol, schwarz_cutoff=1e-12)
        fb.set_shard(r, 3)
        j, k = fb.make_r_JK(P)
        Js += j
        Ks += k
    assert np.max(np.abs(Js - J)) < 1e-12 and np.max(np.abs(Ks - K)) < 1e-12


@pytest.mark.gpu
def test_rhf_energy_matches_oracle_scf(cuda_ok, oracle_mod):
    from tonto_b200.scf import RHF
    mol = water_cluster(3, seed=0)
    ref = oracle_mod.scf(mol, oracle_mod.Oracle(mol, schwarz_cutoff=1e-12), conv=1e-10, diis_tol=1e-7)
    r = RHF(mol, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    assert r.converged
    assert abs(r.energy - ref["E"]) < 1e-9, (r.energy, ref["E"])


@pytest.mark.gpu
def test_fixture_energy_on_gpu(cuda_ok, oracle_mod):
    """Tonto's blessed cc-pVDZ H2O energy (-76.023280, tests/short/h2o_rhf_cc-pVDZ_electron_density_plot)
    from the GPU J/K builder (Cartesian basis, as the fixture)."""
    from tonto_b200.molecules import from_angstrom
    from tonto_b200.scf import RHF
    mol = from_angstrom([8, 1, 1], [[-0.028260, 0, 0], [0.599917, 0.767600, 0], [0.599917, -0.767600, 0]],
                        "cc-pVDZ", spherical=False)
    r = RHF(mol, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    assert abs(r.energy - (-76.023280)) <= 5e-7
