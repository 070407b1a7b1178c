"""The batched SCF driver (size buckets, masks, batched DIIS, purification, fall-back)
on CPU tensors, with the oracle's J/K standing in for the batched CUDA builder: every
molecule converges to the oracle's own SCF energy, with or without the incremental and
mixed-precision schedule."""

import numpy as np
import pytest
import torch

from tonto_b200.batch import BatchRHF
from tonto_b200.molecules import water_cluster


class OracleBatchBuilder:
    """The slice of BatchFockBuilder that BatchRHF uses: per-molecule n x n blocks
    concatenated (row-major blocks; P, J, K are symmetric), J and K from the oracle."""

    def __init__(self, oracle_mod, mols):
        self.orcs = [oracle_mod.Oracle(m, schwarz_cutoff=1e-12) for m in mols]
        self.n = [m.n_bf for m in mols]
        self.offsets = np.concatenate([[0], np.cumsum([n * n for n in self.n])]).astype(np.int64)

    def one_electron(self):
        S, T, V = zip(*(o.one_electron() for o in self.orcs))
        return list(S), list(T), list(V)

    def make_r_JK_device(self, P, J, K, flags=0):
        for o, n, a in zip(self.orcs, self.n, self.offsets):
            Jn, Kn = o.jk(P[a:a + n * n].reshape(n, n).numpy())
            J[a:a + n * n] = torch.from_numpy(np.ascontiguousarray(Jn)).reshape(-1)
            K[a:a + n * n] = torch.from_numpy(np.ascontiguousarray(Kn)).reshape(-1)


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
