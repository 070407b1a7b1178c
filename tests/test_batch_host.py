"""Host-side pieces of the batched SCF driver, on CPU tensors: the purification
that replaces the diagonalisation and the batched DIIS."""

import numpy as np
import torch

from tonto_b200.batch import BatchRHF, purify
from tonto_b200.scf import DIIS


def test_purification_gives_the_aufbau_projector():
    rng = np.random.default_rng(1)
    sizes, n_occ = [7, 12, 9], [3, 5, 4]
    n = max(sizes)
    F = torch.zeros((3, n, n), dtype=torch.float64)
    refs = []
    for k, (m, no) in enumerate(zip(sizes, n_occ)):
        # well separated occupied / virtual levels, like a molecule (gap ~ 0.5)
        e = np.concatenate([rng.uniform(-20.0, -0.6, no), rng.uniform(0.0, 5.0, m - no)])
        Q, _ = np.linalg.qr(rng.normal(size=(m, m)))
        A = Q @ np.diag(e) @ Q.T
        F[k, :m, :m] = torch.tensor(A)
        refs.append(Q[:, :no] @ Q[:, :no].T)
    valid = torch.arange(n)[None, :] < torch.tensor(sizes)[:, None]
    P = purify(F, valid, torch.tensor(n_occ))
    for k, m in enumerate(sizes):
        assert np.max(np.abs(P[k, :m, :m].numpy() - refs[k])) < 1e-11
        assert np.max(np.abs(P[k, m:, :].numpy()), initial=0.0) == 0.0
        assert np.max(np.abs(P[k, :, m:].numpy()), initial=0.0) == 0.0


class _B:
    pass


def test_batched_diis_matches_the_single_diis():
    rng = np.random.default_rng(2)
    m, n, keep = 3, 5, 4
    b = _B()
    b.m = m
    b.Fh = torch.zeros((m, keep, n, n), dtype=torch.float64)
    b.Eh = torch.zeros_like(b.Fh)
    b.count = torch.zeros(m, dtype=torch.long)
    singles = [DIIS(keep) for _ in range(m)]
    for cyc in range(7):
        cm = torch.tensor([True, cyc % 2 == 0, cyc >= 2])
        b.F = torch.tensor(rng.normal(size=(m, n, n)))
        b.err = torch.tensor(rng.normal(size=(m, n, n)))
        Fx = BatchRHF._diis(b, cm, keep)
        for i in range(m):
            if bool(cm[i]):
                ref = singles[i].extrapolate(b.F[i], b.err[i])
                assert torch.max(torch.abs(Fx[i] - ref)) < 1e-10
