"""Moving the atoms of a context (tf_set_geometry), as Hirshfeld-atom refinement does
between SCFs: J/K and one-electron matrices against fresh contexts and the oracle,
and an SCF restarted from the previous geometry's density."""

import dataclasses

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster


def _moved(mol, seed, step=0.05):
    rng = np.random.default_rng(seed)
    return dataclasses.replace(mol, xyz=mol.xyz + rng.uniform(-step, step, size=mol.xyz.shape))


@pytest.mark.gpu
def test_set_geometry_matches_a_fresh_context(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    a = water_cluster(2, seed=12)
    b = _moved(a, 1)
    rng = np.random.default_rng(13)
    A = rng.normal(size=(a.n_bf, a.n_bf)) * 0.05
    P = A + A.T
    fb = FockBuilder(a, schwarz_cutoff=1e-12)
    fb.make_r_JK(P)
    fb.make_r_JK(P)                                  # a captured graph exists for the old geometry
    fb.set_geometry(b.xyz)
    fb.mol = b
    for _ in range(2):
        J, K = fb.make_r_JK(P)
        Jr, Kr = oracle_mod.Oracle(b, schwarz_cutoff=1e-12).jk(P)
        assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11
    S, T, V = fb.one_electron()
    S0, T0, V0 = FockBuilder(b).one_electron()
    for X, Y in ((S, S0), (T, T0), (V, V0)):
        assert np.max(np.abs(X - Y)) < 1e-12


@pytest.mark.gpu
def test_scf_restarted_after_a_move(cuda_ok):
    from tonto_b200.scf import RHF
    a = water_cluster(3, seed=14)
    b = _moved(a, 2, step=0.02)
    rhf = RHF(a, schwarz_cutoff=1e-12)
    ra = rhf.run(conv=1e-10, diis_tol=1e-7)
    rhf.set_geometry(b.xyz)
    rb = rhf.run(P0=ra.P, conv=1e-10, diis_tol=1e-7, guess_name="previous geometry")
    fresh = RHF(b, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    assert rb.converged and abs(rb.energy - fresh.energy) < 1e-9
    assert rb.iterations < fresh.iterations
