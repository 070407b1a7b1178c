"""The SCF side of Hirshfeld-atom refinement (molecule.har.foo:352-491): repeated SCFs
at moved atoms, each from the previous density, and several geometries of one
molecule solved together in one batched context, against fresh SCFs."""

import dataclasses

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster


def _moved(mol, seed, step):
    rng = np.random.default_rng(seed)
    return mol.xyz + rng.uniform(-step, step, size=mol.xyz.shape)


@pytest.mark.gpu
def test_har_cycle_restarts_from_the_previous_density(cuda_ok):
    from tonto_b200.har import HARCycle
    from tonto_b200.scf import RHF
    mol = water_cluster(3, seed=21)
    cyc = HARCycle(mol)
    r0 = cyc.scf(conv=1e-10, diis_tol=1e-7)
    assert r0.converged
    for k in range(2):                            # two refinement steps
        xyz = _moved(mol, 30 + k, 0.02)
        r = cyc.scf(xyz, conv=1e-10, diis_tol=1e-7)
        fresh = RHF(dataclasses.replace(mol, xyz=xyz), schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
        assert r.converged and abs(r.energy - fresh.energy) < 1e-9
        assert r.iterations < fresh.iterations


@pytest.mark.gpu
def test_geometries_solved_together_match_single_scfs(cuda_ok):
    from tonto_b200.har import scf_at_geometries
    from tonto_b200.scf import RHF
    mol = water_cluster(2, seed=22)
    base = RHF(mol, schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
    geoms = [_moved(mol, 40 + k, 0.03) for k in range(4)]
    res = scf_at_geometries(mol, geoms, P0=base.P, conv=1e-10, diis_tol=1e-7)
    cold = []
    for xyz, r in zip(geoms, res):
        fresh = RHF(dataclasses.replace(mol, xyz=xyz), schwarz_cutoff=1e-12).run(conv=1e-10, diis_tol=1e-7)
        cold.append(fresh.iterations)
        assert r.converged and abs(r.energy - fresh.energy) < 1e-9
    assert np.mean([r.iterations for r in res]) < np.mean(cold)
