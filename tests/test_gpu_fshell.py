"""f shells on the GPU path (cc-pVTZ): J, K, unrestricted J, K, Schwarz bounds and
one-electron integrals against the oracle, and Tonto's only spherical RHF fixture
(tests/short/h2o_rhf_cc-pVTZ_spherical_harmonic_basis/stdout:204, E = -76.0524 with
f functions on O) reproduced through the GPU builder.  The classes with an f shell
run the warp kernel (k_jk_warp); Rys quadrature with up to 7 roots for (ff|ff)
(RYS:get_weights, rys.foo:89-134)."""

import json
import os

import numpy as np
import pytest

from tonto_b200.molecules import from_angstrom, water_cluster

TOL = 1e-11
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _core_density(oracle_mod, orc, mol):
    S, T, V = orc.one_electron()
    P, _, _ = oracle_mod.density_from_fock(T + V, oracle_mod.orthogonaliser(S), mol.n_electrons // 2)
    return P


def _class_counts(orc):
    cnt = orc.counts(reset=True).reshape(625, 2)
    sym = "spdfg"
    out = {}
    for q in range(625):
        if cnt[q, 0] > 0:
            l = (q // 125, (q // 25) % 5, (q // 5) % 5, q % 5)
            out["(%s%s|%s%s)" % tuple(sym[v] for v in l)] = (cnt[q, 0], cnt[q, 1])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("spherical", [True, False])
def test_cc_pvtz_jk_matches_oracle(cuda_ok, oracle_mod, spherical):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(2, seed=4, basis="cc-pVTZ", spherical=spherical)
    assert any(s.l == 3 for s in mol.shells)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    rng = np.random.default_rng(7)
    A = rng.normal(size=(mol.n_bf, mol.n_bf)) * 0.02
    for P in (_core_density(oracle_mod, orc, mol), A + A.T):
        fb = FockBuilder(mol, schwarz_cutoff=1e-12)
        fb.set_graph(False)
        J, K = fb.make_r_JK(P)
        got = {c["class"]: (c["quartets"], c["prim_quartets"]) for c in fb.class_stats() if c["quartets"] > 0}
        fb.set_graph(True)
        Jg, Kg = fb.make_r_JK(P)
        Jg, Kg = fb.make_r_JK(P)                   # a replayed graph
        fb.close()
        orc.counts(reset=True)
        Jr, Kr = orc.jk(P)
        assert got == _class_counts(orc)
        assert any("f" in k for k in got)
        for a, b in ((J, Jr), (K, Kr), (Jg, Jr), (Kg, Kr)):
            assert np.max(np.abs(a - b)) <= TOL


@pytest.mark.gpu
def test_cc_pvtz_schwarz_and_one_electron(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    for spherical in (True, False):
        mol = water_cluster(2, seed=5, basis="cc-pVTZ", spherical=spherical)
        orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
        fb = FockBuilder(mol, schwarz_cutoff=1e-12)
        mi, mr = fb.max_I, orc.max_I()
        assert np.max(np.abs(mi - mr) / np.maximum(mr, 1e-300)) <= 1e-12
        S0, T0, V0 = orc.one_electron()
        S, T, V = fb.one_electron()
        for a, b in ((S, S0), (T, T0), (V, V0)):
            assert np.max(np.abs(a - b)) < 1e-11
        fb.close()


@pytest.mark.gpu
def test_cc_pvtz_unrestricted_jk_matches_oracle(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(1, seed=6, basis="cc-pVTZ")
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    rng = np.random.default_rng(3)
    A = rng.normal(size=(mol.n_bf, mol.n_bf)) * 0.03
    B = rng.normal(size=(mol.n_bf, mol.n_bf)) * 0.03
    Pa, Pb = A + A.T, B + B.T
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    got = fb.make_u_JK(Pa, Pb)
    ref = orc.jk_uhf(Pa, Pb)
    for a, b in zip(got, ref):
        assert np.max(np.abs(a - b)) <= TOL


@pytest.mark.gpu
def test_cc_pvtz_fixture_on_gpu(cuda_ok, oracle_mod):
    """Tonto's blessed spherical cc-pVTZ water: every printed energy term from the GPU
    J/K build (to Tonto's gate, two units in the last printed digit; the blessed SCF
    stopped at |dE| < 1e-5, so E itself to half a unit), and the converged energy
    within 1e-9 Eh of the oracle SCF."""
    import torch
    from tonto_b200.scf import RHF
    with open(os.path.join(GOLD, "tonto_fixtures.json")) as fh:
        case = [c for c in json.load(fh)["cases"] if c["case"] == "h2o_rhf_cc-pVTZ_spherical_harmonic_basis"][0]
    Z = [a[0] for a in case["atoms_angstrom"]]
    xyz = [a[1:] for a in case["atoms_angstrom"]]
    mol = from_angstrom(Z, xyz, case["basis"], spherical=case["spherical"])
    assert mol.n_bf == case["n_bf"] == 58
    rhf = RHF(mol, schwarz_cutoff=1e-12)
    r = rhf.run(conv=1e-10, diis_tol=1e-7)
    assert r.converged
    P = r.P
    J, K = rhf.jk(P)
    terms = {"E": r.energy, "V_NN": rhf.e_nuc, "T": float(torch.sum(P * rhf.T)), "V_eN": float(torch.sum(P * rhf.V)),
             "V_ee": 0.5 * float(torch.sum(P * (J - 0.5 * K)))}
    for key, ref in case["results"].items():
        ulp = 10.0 ** (-ref["decimals"])
        tol = (0.5 + 1e-6) * ulp if key == "E" else 2.0 * ulp
        assert abs(terms[key] - ref["value"]) <= tol, (key, terms[key], ref["value"])
    ref_scf = oracle_mod.scf(mol, oracle_mod.Oracle(mol, schwarz_cutoff=1e-12), conv=1e-10, diis_tol=1e-7)
    assert abs(r.energy - ref_scf["E"]) < 1e-9
