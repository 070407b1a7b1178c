"""The oracle's screening and primitive counting against a plain numpy statement of
Tonto's rules (molecule.fock.foo:1274-1318, 3454-3495): a quartet (ab|cd), cd <= ab in
pair order, is computed when I_max(ab) I_max(cd) max|P| over the six shell-pair blocks
exceeds the cutoff and that maximum is at least 1e-20; its primitive quartets are the
products of all primitive pairs when any two of its atoms coincide, else of the pairs with
exp(-ab R^2 / zeta) >= 1e-6.  (On the GPU, the library's per-build counts equal the
oracle's: 359,071,641 quartets and 3,563,474,977 primitive quartets for (H2O)32 at its
core-guess density.)"""

import numpy as np

from tonto_b200.molecules import water_cluster


def _counts(mol, Imax, P, cutoff):
    sh = mol.shells
    ns = len(sh)
    f0 = np.array([s.first_bf for s in sh])
    pm = np.maximum.reduceat(np.maximum.reduceat(np.abs(P), f0, axis=0), f0, axis=1)
    atom = np.array([s.atom for s in sh])
    pa = np.concatenate([np.full(a + 1, a) for a in range(ns)])
    pb = np.concatenate([np.arange(a + 1) for a in range(ns)])
    nfull = np.array([len(sh[a].exps) * len(sh[b].exps) for a, b in zip(pa, pb)])
    nskip = nfull.copy()
    for p, (a, b) in enumerate(zip(pa, pb)):
        if atom[a] != atom[b]:
            R2 = float(np.sum((mol.xyz[atom[a]] - mol.xyz[atom[b]]) ** 2))
            ea, eb = np.array(sh[a].exps)[:, None], np.array(sh[b].exps)[None, :]
            nskip[p] = int(np.sum(np.exp(-ea * eb / (ea + eb) * R2) >= 1e-6))
    nq = npq = 0
    for p in range(len(pa)):
        a, b = pa[p], pb[p]
        c, d = pa[:p + 1], pb[:p + 1]
        m = np.maximum.reduce([np.full(p + 1, pm[a, b]), pm[c, d], pm[a, c], pm[a, d], pm[b, c], pm[b, d]])
        ok = (Imax[p] * Imax[:p + 1] * m > cutoff) & (m >= 1e-20)
        idx = np.flatnonzero(ok)
        ca, da = atom[pa[idx]], atom[pb[idx]]
        same = ((atom[a] == atom[b]) | (ca == da) | (atom[a] == ca) | (atom[a] == da)
                | (atom[b] == ca) | (atom[b] == da))
        nq += len(idx)
        npq += int(np.where(same, nfull[p] * nfull[idx], nskip[p] * nskip[idx]).sum())
    return nq, npq


def test_oracle_screening_and_primitive_counts(oracle_mod):
    mol = water_cluster(4, seed=0)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    S, T, V = orc.one_electron()
    P = oracle_mod.density_from_fock(T + V, oracle_mod.orthogonaliser(S), mol.n_electrons // 2)[0]
    rng = np.random.default_rng(3)
    A = rng.normal(size=P.shape) * 1e-3
    for D in (P, A + A.T):                        # a density and a small density change
        orc.counts(reset=True)
        orc.jk(D)
        c = orc.counts()
        nq, npq = _counts(mol, orc.max_I(), D, 1e-12)
        assert int(c[..., 0].sum()) == nq and int(c[..., 1].sum()) == npq
