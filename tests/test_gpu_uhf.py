"""Unrestricted J/K (make_u_JK_direct) and the J-only / K-only builds against the
oracle; UHF SCF against the oracle's UHF."""

import numpy as np
import pytest

from tonto_b200.molecules import from_angstrom, water_cluster


def _sym(rng, n, s):
    A = rng.normal(size=(n, n)) * s
    return A + A.T


@pytest.mark.gpu
def test_uhf_jk_matches_oracle(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder, TF_JK_MIXED
    mol = water_cluster(2, seed=3)
    rng = np.random.default_rng(21)
    Pa, Pb = _sym(rng, mol.n_bf, 0.05), _sym(rng, mol.n_bf, 0.04)
    ref = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk_uhf(Pa, Pb)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    out = fb.make_u_JK(Pa, Pb)
    for X, Y in zip(out, ref):
        assert np.max(np.abs(X - Y)) < 1e-11
    out32 = fb.make_u_JK(Pa, Pb, TF_JK_MIXED)
    for X, Y in zip(out32, ref):
        assert np.max(np.abs(X - Y)) < 1e-8
    # the restricted build is untouched by an unrestricted one on the same context
    J, K = fb.make_r_JK(Pa + Pb)
    Jr, Kr = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk(Pa + Pb)
    assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11


@pytest.mark.gpu
def test_j_only_and_k_only(cuda_ok):
    from tonto_b200.fock import FockBuilder, TF_JK_J_ONLY, TF_JK_K_ONLY
    mol = water_cluster(3, seed=4)
    rng = np.random.default_rng(22)
    P = _sym(rng, mol.n_bf, 0.05)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    J, K = fb.make_r_JK(P)
    for _ in range(2):                          # direct build, then the captured graph
        Jj, Kj = fb.make_r_JK(P, TF_JK_J_ONLY)
        assert np.max(np.abs(Jj - J)) < 1e-12 and np.max(np.abs(Kj)) == 0.0
        Jk, Kk = fb.make_r_JK(P, TF_JK_K_ONLY)
        assert np.max(np.abs(Kk - K)) < 1e-12 and np.max(np.abs(Jk)) == 0.0
    with pytest.raises(Exception):
        fb.make_r_JK(P, TF_JK_J_ONLY | TF_JK_K_ONLY)


@pytest.mark.gpu
def test_uhf_scf_matches_oracle(cuda_ok, oracle_mod):
    from tonto_b200.scf import RHF, UHF
    oh = from_angstrom([8, 1], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.97]]), "cc-pVDZ", True)
    u = UHF(oh, multiplicity=2, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    ref = oracle_mod.uhf_scf(oh, 5, 4, oracle_mod.Oracle(oh, schwarz_cutoff=1e-12), conv=1e-10, diis_tol=1e-7)
    assert u.converged and abs(u.energy - ref["E"]) < 1e-9
    w = water_cluster(1, seed=0)
    r = RHF(w, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    uw = UHF(w, multiplicity=1, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    assert abs(uw.energy - r.energy) < 1e-9
