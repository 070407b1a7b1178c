"""Batched contexts: many molecules per build, checked molecule by molecule."""

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster


@pytest.mark.gpu
def test_batched_build_matches_single_builds(cuda_ok, oracle_mod):
    from tonto_b200.fock import BatchFockBuilder, FockBuilder, TF_JK_MIXED
    mols = [water_cluster(n, seed=20 + n) for n in (2, 3, 1, 4)]
    rng = np.random.default_rng(3)
    Ps = []
    for m in mols:
        A = rng.normal(size=(m.n_bf, m.n_bf)) * 0.05
        Ps.append(A + A.T)
    bb = BatchFockBuilder(mols, schwarz_cutoff=1e-12)
    Js, Ks = bb.make_r_JK_batched(Ps)
    for m, P, J, K in zip(mols, Ps, Js, Ks):
        Jr, Kr = oracle_mod.Oracle(m, schwarz_cutoff=1e-12).jk(P)
        assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11
    # one-electron integrals per molecule
    S, T, V = bb.one_electron()
    for i, m in enumerate(mols):
        S0, T0, V0 = FockBuilder(m).one_electron()
        assert np.max(np.abs(S[i] - S0)) < 1e-12 and np.max(np.abs(V[i] - V0)) < 1e-11
    # the batch in mixed precision stays within the FP32 error bound
    Jm, Km = bb.make_r_JK_batched(Ps, TF_JK_MIXED)
    assert max(float(np.max(np.abs(a - b))) for a, b in zip(Jm, Js)) < 1e-8
    # quartet lists written and consumed in small chunks (many class-pair chunks,
    # some class pairs alone larger than the budget) give the same J and K
    total = int(bb.stats()["quartets"])
    for budget in (total // 7, 1000):
        bb.set_list_budget(budget)
        Jc, Kc = bb.make_r_JK_batched(Ps)
        assert int(bb.stats()["quartets"]) == total
        for a, b in zip(Jc + Kc, Js + Ks):
            assert np.max(np.abs(a - b)) < 1e-12


@pytest.mark.gpu
def test_batched_scf_matches_single_scf(cuda_ok):
    from tonto_b200.batch import BatchRHF
    from tonto_b200.scf import RHF
    mols = [water_cluster(n, seed=40 + n) for n in (2, 3, 4)]
    res = BatchRHF(mols, schwarz_cutoff=1e-12).run(conv=1e-9, diis_tol=1e-6)
    for m, r in zip(mols, res):
        ref = RHF(m, schwarz_cutoff=1e-12).run(conv=1e-9, diis_tol=1e-6)
        assert r.converged and abs(r.energy - ref.energy) < 1e-8


@pytest.mark.gpu
def test_per_molecule_cutoffs_screen_each_molecule_on_its_own(cuda_ok, oracle_mod):
    """tf_set_molecule_cutoffs: each molecule of a batched build is screened with its
    own Schwarz x density cutoff, exactly as a single-molecule context with that cutoff
    (the same quartets, J and K against the oracle at that cutoff), class by class and
    in replayed graph builds whose cutoffs change between replays."""
    from tonto_b200.fock import BatchFockBuilder, FockBuilder
    mols = [water_cluster(n, seed=60 + n) for n in (3, 2, 4)]
    rng = np.random.default_rng(9)
    Ps = []
    for m in mols:
        A = rng.normal(size=(m.n_bf, m.n_bf)) * 0.05
        Ps.append(A + A.T)
    bb = BatchFockBuilder(mols, schwarz_cutoff=1e-12)
    for graph in (False, True):
        bb.set_graph(graph)
        for cuts in ([1e-12, 1e-8, 1e-10], [1e-9, 1e-12, 1e-7]):
            bb.set_molecule_cutoffs(cuts)
            for _ in range(2 if graph else 1):              # capture, then replay
                Js, Ks = bb.make_r_JK_batched(Ps)
            quartets = 0
            for m, P, J, K, c in zip(mols, Ps, Js, Ks, cuts):
                Jr, Kr = oracle_mod.Oracle(m, schwarz_cutoff=c).jk(P)
                assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11
                f = FockBuilder(m, schwarz_cutoff=c)
                f.make_r_JK(P)
                quartets += int(f.stats()["quartets"])
                f.close()
            assert int(bb.stats()["quartets"]) == quartets
    bb.set_molecule_cutoffs(None)                            # back to the context's cutoff
    Js, Ks = bb.make_r_JK_batched(Ps)
    for m, P, J, K in zip(mols, Ps, Js, Ks):
        Jr, Kr = oracle_mod.Oracle(m, schwarz_cutoff=1e-12).jk(P)
        assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11
    with pytest.raises(Exception):
        bb.set_molecule_cutoffs([1e-12, -1.0, 1e-12])
    with pytest.raises(ValueError):
        bb.set_molecule_cutoffs([1e-12, 1e-12])
    bb.close()
