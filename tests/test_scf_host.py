"""The SCF driver's control flow on CPU tensors, with the oracle's J/K standing in for
the CUDA builder: the cheap state (incremental builds of the density change), the
switch to full FP64 builds near convergence (final_at), the two final full builds, and
the fall-back to a second guess.  The converged energy must not depend on any of it."""

import types

import numpy as np
import pytest
import torch

from tonto_b200.molecules import water_cluster
from tonto_b200.scf import RHF


class OracleBuilder:
    """The slice of FockBuilder that RHF uses, computed by the oracle (all flags give
    FP64; TF_JK_DELTA needs nothing, J and K being linear in the density)."""

    def __init__(self, oracle_mod, mol):
        self.o = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
        self.options = types.SimpleNamespace(eri_schwarz_cutoff=1e-12)
        self.builds = 0

    def one_electron(self):
        return self.o.one_electron()

    def make_r_JK_device(self, P, J, K, flags=0):
        Jn, Kn = self.o.jk(P.numpy())
        J.copy_(torch.from_numpy(np.ascontiguousarray(Jn)))
        K.copy_(torch.from_numpy(np.ascontiguousarray(Kn)))
        self.builds += 1

    def set_schwarz_cutoff(self, cut):
        pass


@pytest.fixture(scope="module")
def water2(oracle_mod):
    mol = water_cluster(2, seed=1)
    ref = oracle_mod.scf(mol, conv=1e-9, diis_tol=1e-6)
    return mol, ref


def test_plain_run_matches_the_oracle_scf(oracle_mod, water2):
    mol, ref = water2
    rhf = RHF(mol, device=torch.device("cpu"), builder=OracleBuilder(oracle_mod, mol))
    r = rhf.run(conv=1e-9, diis_tol=1e-6)
    assert r.converged and abs(r.energy - ref["E"]) < 1e-9
    assert r.builds == r.iterations + 1
    assert all(h[4] == "fp64" for h in r.history)


def test_incremental_run_ends_with_full_fp64_builds(oracle_mod, water2):
    mol, ref = water2
    cpu = torch.device("cpu")
    plain = RHF(mol, device=cpu, builder=OracleBuilder(oracle_mod, mol)).run(conv=1e-9, diis_tol=1e-6)
    fast = RHF(mol, device=cpu, builder=OracleBuilder(oracle_mod, mol)).run(
        conv=1e-9, diis_tol=1e-6, mixed=True, incremental=True)
    assert fast.converged and abs(fast.energy - ref["E"]) < 1e-9
    kinds = [h[4] for h in fast.history]
    assert kinds[0] == "mixed" and any(k.endswith("+delta") for k in kinds)
    assert kinds[-2:] == ["fp64", "fp64"]                      # the last two builds full FP64
    # the switch comes once the DIIS error is within final_at x tolerance, so the
    # final builds fall on cycles the plain SCF needs as well
    first_full = kinds.index("fp64", 1)
    assert fast.history[first_full - 1][3] < 10.0 * 1e-6
    assert fast.builds <= plain.builds + 1


def test_fallback_replaces_a_guess_that_does_not_converge(oracle_mod, water2):
    mol, ref = water2
    rhf = RHF(mol, device=torch.device("cpu"), builder=OracleBuilder(oracle_mod, mol))
    n = mol.n_bf
    # a zero density commutes with the core Fock matrix (DIIS error 0), so the error can
    # only grow from the first cycle: the fall-back must replace it
    bad = torch.zeros((n, n), dtype=torch.float64)
    good = rhf.core_guess()
    r = rhf.run(P0=bad, conv=1e-9, diis_tol=1e-6, fallback=lambda: good, fallback_after=1)
    assert r.fell_back
    assert r.converged and abs(r.energy - ref["E"]) < 1e-9


class CutoffOracleBuilder(OracleBuilder):
    """OracleBuilder whose builds honour the Schwarz cutoff set last (one oracle per
    cutoff value), recording the cutoff of every build."""

    def __init__(self, oracle_mod, mol):
        super().__init__(oracle_mod, mol)
        self.mod, self.mol = oracle_mod, mol
        self.by_cut = {1e-12: self.o}
        self.cuts = []
        self.mol_cut = None

    def set_schwarz_cutoff(self, cut):
        self.options.eri_schwarz_cutoff = cut

    def make_r_JK_device(self, P, J, K, flags=0):
        cut = self.mol_cut if self.mol_cut is not None else self.options.eri_schwarz_cutoff
        if cut not in self.by_cut:
            self.by_cut[cut] = self.mod.Oracle(self.mol, schwarz_cutoff=cut)
        self.o = self.by_cut[cut]
        self.cuts.append(cut)
        super().make_r_JK_device(P, J, K, flags)


class MolCutoffOracleBuilder(CutoffOracleBuilder):
    """The same with a per-molecule cutoff (one molecule), as the CUDA builder offers."""

    def set_molecule_cutoffs(self, cuts):
        self.mol_cut = None if cuts is None else float(cuts[0])


@pytest.mark.parametrize("builder", [CutoffOracleBuilder, MolCutoffOracleBuilder])
def test_loosened_cheap_cycles_keep_the_converged_energy(oracle_mod, water2, builder):
    """Cheap cycles with a Schwarz cutoff that follows the DIIS error (loosen x error,
    clamped to [tight, loose_max]), set as the context cutoff or as the molecule's own
    cutoff; the final full builds at the tight cutoff decide the energy, which stays the
    oracle's."""
    mol, ref = water2
    fb = builder(oracle_mod, mol)
    r = RHF(mol, device=torch.device("cpu"), builder=fb).run(conv=1e-9, diis_tol=1e-6, incremental=True,
                                                            loosen=1e-4, loose_max=1e-8)
    assert r.converged and abs(r.energy - ref["E"]) < 1e-9
    kinds = [h[4] for h in r.history]
    assert fb.cuts[0] == 1e-8                                   # first build: the loosest cutoff
    for cut, kind, h_prev in zip(fb.cuts[1:], kinds[1:], r.history[:-1]):
        if kind.endswith("+delta"):
            assert cut == min(1e-8, max(1e-12, 1e-4 * h_prev[3]))
    assert fb.cuts[-2:] == [1e-12, 1e-12] and kinds[-2:] == ["fp64", "fp64"]
    assert any(c > 1e-12 for c in fb.cuts[1:-2])
    assert fb.options.eri_schwarz_cutoff == 1e-12 and fb.mol_cut is None   # restored after the run


class OracleUBuilder(OracleBuilder):
    """Adds the unrestricted build (make_u_JK_direct) from the oracle."""

    def make_u_JK_device(self, Pa, Pb, Ja, Jb, Ka, Kb, flags=0):
        out = self.o.jk_uhf(Pa.numpy(), Pb.numpy())
        for t, a in zip((Ja, Jb, Ka, Kb), out):
            t.copy_(torch.from_numpy(np.ascontiguousarray(a)))


def test_uhf_driver_matches_the_oracle_uhf(oracle_mod):
    from tonto_b200.molecules import from_angstrom
    from tonto_b200.scf import UHF
    oh = from_angstrom([8, 1], np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.97]]), "cc-pVDZ", True)
    ref = oracle_mod.uhf_scf(oh, 5, 4, conv=1e-9, diis_tol=1e-6)
    u = UHF(oh, multiplicity=2, device=torch.device("cpu"), builder=OracleUBuilder(oracle_mod, oh))
    r = u.run(conv=1e-9, diis_tol=1e-6)
    assert r.converged and abs(r.energy - ref["E"]) < 1e-9
