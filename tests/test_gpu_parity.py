"""GPU J/K against the oracle (Tonto's make_r_JK_direct / make_r_JK_engine restated).

Bar: max |J - J_ref|, max |K - K_ref| <= 1e-11 per element (FP64 path), on the
same density and the same Schwarz and primitive-pair cutoffs.
"""

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster, alkane, from_angstrom

TOL = 1e-11


def core_density(orc, oracle_mod, mol):
    S, T, V = orc.one_electron()
    X = oracle_mod.orthogonaliser(S)
    P, _, _ = oracle_mod.density_from_fock(T + V, X, mol.n_electrons // 2)
    return P


def compare(mol, oracle_mod, schwarz=1e-12, P=None):
    from tonto_b200.fock import FockBuilder
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=schwarz)
    if P is None:
        P = core_density(orc, oracle_mod, mol)
    Jr, Kr = orc.jk(P)
    fb = FockBuilder(mol, schwarz_cutoff=schwarz)
    J, K = fb.make_r_JK(P)
    dj = float(np.max(np.abs(J - Jr)))
    dk = float(np.max(np.abs(K - Kr)))
    return dj, dk, fb, orc


@pytest.mark.gpu
@pytest.mark.parametrize("spherical", [True, False])
def test_water_dimer(cuda_ok, oracle_mod, spherical):
    mol = water_cluster(2, seed=7, spherical=spherical)
    dj, dk, fb, orc = compare(mol, oracle_mod)
    assert dj <= TOL and dk <= TOL, (dj, dk)


@pytest.mark.gpu
def test_water_tetramer_core_guess(cuda_ok, oracle_mod):
    mol = water_cluster(4, seed=0)
    assert mol.n_bf == 96
    dj, dk, fb, orc = compare(mol, oracle_mod)
    assert dj <= TOL and dk <= TOL, (dj, dk)


@pytest.mark.gpu
def test_schwarz_bounds_match(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(3, seed=2)
    orc = oracle_mod.Oracle(mol)
    fb = FockBuilder(mol)
    a, b = fb.max_I, orc.max_I()
    assert np.max(np.abs(a - b) / np.maximum(b, 1e-300)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("basis", ["STO-3G", "6-31G(d)", "def2-SVP"])
def test_other_bases(cuda_ok, oracle_mod, basis):
    mol = water_cluster(2, seed=11, basis=basis)
    dj, dk, fb, orc = compare(mol, oracle_mod, schwarz=1e-10)
    assert dj <= TOL and dk <= TOL, (dj, dk)


@pytest.mark.gpu
def test_small_alkane_def2svp(cuda_ok, oracle_mod):
    mol = alkane(4, seed=0)
    dj, dk, fb, orc = compare(mol, oracle_mod)
    assert dj <= TOL and dk <= TOL, (dj, dk)


@pytest.mark.gpu
def test_random_symmetric_density(cuda_ok, oracle_mod):
    mol = water_cluster(2, seed=5)
    rng = np.random.default_rng(0)
    A = rng.normal(size=(mol.n_bf, mol.n_bf)) * 0.1
    P = A + A.T
    dj, dk, fb, orc = compare(mol, oracle_mod, P=P)
    assert dj <= TOL and dk <= TOL, (dj, dk)


@pytest.mark.gpu
def test_fock_matches_j_minus_half_k(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(2, seed=4)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P = core_density(orc, oracle_mod, mol)
    S, T, V = orc.one_electron()
    H = T + V
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    F = fb.make_r_Fock_mx(P, H)
    Jr, Kr = orc.jk(P)
    assert np.max(np.abs(F - (H + Jr - 0.5 * Kr))) <= TOL


@pytest.mark.gpu
@pytest.mark.parametrize("n_water", [4, 12])
def test_mixed_precision_build_error_is_bounded(cuda_ok, oracle_mod, n_water):
    """TF_JK_MIXED: quartets whose Schwarz x density bound is below the cut (1e-6) are
    evaluated in FP32 after FP64 Rys nodes and weights, and accumulated in FP64.
    The FP32 quartets are the oracle's quartets below the cut, less at most 3 % that
    share a bra-family entry with an above-cut quartet (the count pins the cut), and
    every J, K element is within DELTA of its FP32 error budget of the FP64
    oracle: the budget is the oracle's per-element sum of the bounds of the terms it
    receives from those quartets (|(ab|cd) P| <= bound per term), DELTA a relative
    error of FP32 evaluation, 2^-14, with room for the chain of about fifty FP32
    operations and the spherical transform.  The observed error is far inside it, below
    1e-9, which is checked too."""
    from tonto_b200.fock import FockBuilder, TF_JK_MIXED
    DELTA = 2.0 ** -14
    mol = water_cluster(n_water, seed=0)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P = core_density(orc, oracle_mod, mol)
    Jr, Kr = orc.jk(P)
    Jb, Kb, n32 = orc.fp32_bound(P, 1e-6)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12, mixed_fp32_cut=1e-6)
    J, K = fb.make_r_JK(P, TF_JK_MIXED)
    st = fb.stats()
    assert st["quartets_fp32"] > 0.3 * st["quartets"]
    # a bra-family entry runs in FP32 only when every member quartet it holds is below
    # the cut, so the FP32 member quartets are the oracle's below-cut quartets less the
    # few that share an entry with an above-cut one
    assert 0.97 * n32 <= st["quartets_fp32"] <= n32, (st["quartets_fp32"], n32)
    assert np.all(np.abs(J - Jr) <= DELTA * Jb + 1e-12)
    assert np.all(np.abs(K - Kr) <= DELTA * Kb + 1e-12)
    # and, as observed, far inside that budget
    assert np.max(np.abs(J - Jr)) < 1e-9 and np.max(np.abs(K - Kr)) < 1e-9


@pytest.mark.gpu
def test_delta_build_is_linear(cuda_ok, oracle_mod):
    """TF_JK_DELTA: J, K of a density difference; G[P1] = G[P0] + G[P1 - P0]."""
    from tonto_b200.fock import FockBuilder, TF_JK_DELTA
    mol = water_cluster(2, seed=8)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P0 = core_density(orc, oracle_mod, mol)
    rng = np.random.default_rng(2)
    A = rng.normal(size=P0.shape) * 1e-3
    P1 = P0 + A + A.T
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    J0, K0 = fb.make_r_JK(P0)
    dJ, dK = fb.make_r_JK(P1 - P0, TF_JK_DELTA)
    J1r, K1r = orc.jk(P1)
    assert np.max(np.abs(J0 + dJ - J1r)) < 1e-10 and np.max(np.abs(K0 + dK - K1r)) < 1e-10


@pytest.mark.gpu
def test_host_build_into_caller_arrays(cuda_ok, oracle_mod):
    """make_r_JK(P, out=(J, K)) writes into the caller's Fortran-ordered arrays (here
    views of page-locked buffers, as the end-to-end measurement uses): the same J and K
    as new arrays, within the bar of the oracle."""
    import torch
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(2, seed=7)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P = core_density(orc, oracle_mod, mol)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    n = mol.n_bf
    pin = [torch.empty((n, n), dtype=torch.float64, pin_memory=True) for _ in range(3)]
    pin[0].copy_(torch.from_numpy(np.ascontiguousarray(P.T)))
    out = (pin[1].numpy().T, pin[2].numpy().T)
    J, K = fb.make_r_JK(pin[0].numpy().T, out=out)
    assert J is out[0] and K is out[1]
    J2, K2 = fb.make_r_JK(P)
    assert np.max(np.abs(J - J2)) <= 1e-13 and np.max(np.abs(K - K2)) <= 1e-13     # atomics: same to rounding
    Jr, Kr = orc.jk(P)
    assert np.max(np.abs(J - Jr)) <= TOL and np.max(np.abs(K - Kr)) <= TOL
    with pytest.raises(ValueError):
        fb.make_r_JK(P, out=(np.empty((n, n)), np.empty((n, n))))       # C-ordered: refused
    fb.close()
