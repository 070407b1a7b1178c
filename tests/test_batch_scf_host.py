"""The batched SCF driver (size buckets, masks, batched DIIS, purification, fall-back)
on CPU tensors, with the oracle's J/K standing in for the batched CUDA builder: every
molecule converges to the oracle's own SCF energy, with or without the incremental and
mixed-precision schedule."""

import types

import numpy as np
import pytest
import torch

from tonto_b200.batch import BatchRHF
from tonto_b200.molecules import water_cluster


class OracleBatchBuilder:
    """The slice of BatchFockBuilder that BatchRHF uses: per-molecule n x n blocks
    concatenated (row-major blocks; P, J, K are symmetric), J and K from the oracle."""

    def __init__(self, oracle_mod, mols):
        self.mod, self.mols = oracle_mod, mols
        self.by_cut = {}
        self.orcs = self._oracles(1e-12)
        self.options = types.SimpleNamespace(eri_schwarz_cutoff=1e-12)
        self.cuts = []
        self.mol_cuts = None
        self.n = [m.n_bf for m in mols]
        self.offsets = np.concatenate([[0], np.cumsum([n * n for n in self.n])]).astype(np.int64)

    def _oracles(self, cut):
        if cut not in self.by_cut:
            self.by_cut[cut] = [self.mod.Oracle(m, schwarz_cutoff=cut) for m in self.mols]
        return self.by_cut[cut]

    def set_schwarz_cutoff(self, cut):
        self.options.eri_schwarz_cutoff = cut

    def set_molecule_cutoffs(self, cuts):
        self.mol_cuts = None if cuts is None else [float(c) for c in cuts]

    def one_electron(self):
        S, T, V = zip(*(o.one_electron() for o in self.orcs))
        return list(S), list(T), list(V)

    def make_r_JK_device(self, P, J, K, flags=0):
        cuts = self.mol_cuts or [self.options.eri_schwarz_cutoff] * len(self.mols)
        self.cuts.append(list(cuts))
        orcs = [self._oracles(c)[i] for i, c in enumerate(cuts)]
        for o, n, a in zip(orcs, self.n, self.offsets):
            Jn, Kn = o.jk(P[a:a + n * n].reshape(n, n).numpy())
            J[a:a + n * n] = torch.from_numpy(np.ascontiguousarray(Jn)).reshape(-1)
            K[a:a + n * n] = torch.from_numpy(np.ascontiguousarray(Kn)).reshape(-1)


class GlobalCutoffBatchBuilder(OracleBatchBuilder):
    """A builder with one Schwarz cutoff per build (no per-molecule cutoffs)."""

    def __getattribute__(self, name):
        if name == "set_molecule_cutoffs":
            raise AttributeError(name)
        return super().__getattribute__(name)


@pytest.fixture(scope="module")
def clusters(oracle_mod):
    mols = [water_cluster(1, seed=2), water_cluster(2, seed=1), water_cluster(2, seed=3)]
    refs = [oracle_mod.scf(m, conv=1e-9, diis_tol=1e-6)["E"] for m in mols]
    return mols, refs


@pytest.mark.parametrize("fast", [False, True])
def test_batched_scf_reaches_the_oracle_energies(oracle_mod, clusters, fast):
    mols, refs = clusters
    b = BatchRHF(mols, device=torch.device("cpu"), n_buckets=2, builder=OracleBatchBuilder(oracle_mod, mols))
    res = b.run(conv=1e-9, diis_tol=1e-6, mixed=fast, incremental=fast)
    for r, e in zip(res, refs):
        assert r.converged and abs(r.energy - e) < 1e-9
        if fast:
            kinds = [h[4] for h in r.history]
            assert any(k.endswith("+delta") for k in kinds)
            assert [k.split("+")[0] for k in kinds[-2:]] == ["fp64", "fp64"]
            assert not kinds[-1].endswith("+delta") and not kinds[-2].endswith("+delta")


def test_batched_fallback_replaces_one_molecules_guess(oracle_mod, clusters):
    mols, refs = clusters
    b = BatchRHF(mols, device=torch.device("cpu"), n_buckets=2, builder=OracleBatchBuilder(oracle_mod, mols))
    n1 = mols[1].n_bf
    core = {}                                                    # core guesses, unpadded
    for B in b.buckets:
        D = b.densities(B, B.H)
        for k, i in enumerate(B.ids):
            core[i] = D[k, :mols[i].n_bf, :mols[i].n_bf].clone()
    P0 = [core[i] for i in range(len(mols))]
    P0[1] = torch.zeros((n1, n1), dtype=torch.float64)          # error 0 at first: can only grow
    res = b.run(P0=P0, conv=1e-9, diis_tol=1e-6, incremental=True, fallback_after=1,
                fallback=lambda i: core[i])
    assert res[1].fell_back and not res[0].fell_back and not res[2].fell_back
    for r, e in zip(res, refs):
        assert r.converged and abs(r.energy - e) < 1e-9


def _final_builds(res, n_builds):
    """Per build, the molecules whose build is a final full FP64 one (a full,
    non-incremental build after their first)."""
    n_full = [0] * len(res)
    out = []
    for k in range(n_builds):
        fin = set()
        for i, r in enumerate(res):
            if k < len(r.history) and not r.history[k][4].endswith("+delta"):
                n_full[i] += 1
                if n_full[i] > 1:
                    fin.add(i)
        out.append(fin)
    return out


@pytest.mark.parametrize("per_molecule", [True, False])
def test_batched_loosened_cheap_cycles_keep_the_energies(oracle_mod, clusters, per_molecule):
    """The batch's cheap cycles screen with loosen x DIIS error as the Schwarz cutoff,
    clamped to [tight, loose_max]: per molecule when the builder takes per-molecule
    cutoffs (a molecule in its final full FP64 builds at the tight cutoff, the others
    loosened), else one cutoff per build (the least error of the active molecules, the
    tight one once any molecule is final).  Every energy is still the oracle's."""
    mols, refs = clusters
    fb = (OracleBatchBuilder if per_molecule else GlobalCutoffBatchBuilder)(oracle_mod, mols)
    assert hasattr(fb, "set_molecule_cutoffs") == per_molecule
    b = BatchRHF(mols, device=torch.device("cpu"), n_buckets=2, builder=fb)
    res = b.run(conv=1e-9, diis_tol=1e-6, mixed=True, incremental=True, loosen=1e-4, loose_max=1e-8)
    for r, e in zip(res, refs):
        assert r.converged and abs(r.energy - e) < 1e-9
    assert all(c == 1e-8 for c in fb.cuts[0])
    assert all(1e-12 <= c <= 1e-8 for cuts in fb.cuts for c in cuts)
    assert any(1e-12 < c < 1e-8 for cuts in fb.cuts for c in cuts)
    assert fb.options.eri_schwarz_cutoff == 1e-12 and fb.mol_cuts is None
    finals = _final_builds(res, len(fb.cuts))
    for k, (cuts, fin) in enumerate(zip(fb.cuts, finals)):
        for i in fin:
            assert cuts[i] == 1e-12                          # final builds: the tight cutoff
        if per_molecule and k > 0:
            for i, r in enumerate(res):                      # cheap molecules: their own error
                if k < len(r.history) and i not in fin and r.history[k][4].endswith("+delta"):
                    assert cuts[i] == min(1e-8, max(1e-12, 1e-4 * r.history[k - 1][3]))
        if not per_molecule and fin:
            assert all(c == 1e-12 for c in cuts)
