"""The SCF side of a Hirshfeld-atom-refinement cycle on the GPU builder.

Tonto's HAR (molecule.har.foo:352-491) runs an SCF, fits the atoms against the
structure factors (LS_fit_Hirshfeld_atoms, :437), and runs the SCF again at the
moved atoms until the fit converges (:429-471), every SCF starting from the
previous one's density ("always use initial_density").  The fit itself is outside
the Fock-build path; what the builder serves is the repeated SCF:

* ``HARCycle.scf(xyz)`` — one molecule: the context is moved (tf_set_geometry,
  pair data and Schwarz bounds rebuilt), the one-electron matrices recomputed, and
  the SCF restarted from the last converged density, with incremental builds.
* ``scf_at_geometries(mol, xyz_list, P0)`` — several geometries of one molecule
  at once (trial steps of a line search, or the displaced geometries of a
  finite-difference derivative of the fit), as one batched context: every cycle
  is one J/K launch sequence over all of them, each SCF started from P0.
"""

from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence

import numpy as np
import torch

from .basis import Molecule
from .batch import BatchRHF
from .scf import RHF, SCFResult


class HARCycle:
    """Repeated SCFs of one molecule at moved atoms, each from the previous density."""

    def __init__(self, mol: Molecule, schwarz_cutoff: float = 1e-12, device: int = 0):
        self.rhf = RHF(mol, schwarz_cutoff=schwarz_cutoff, device=device)
        self.P: Optional[torch.Tensor] = None

    def scf(self, xyz_bohr: Optional[np.ndarray] = None, **run_kw) -> SCFResult:
        """The SCF at xyz (bohr; None: the current atoms), started from the last
        converged density when there is one."""
        if xyz_bohr is not None:
            self.rhf.set_geometry(xyz_bohr)
        kw = dict(incremental=True)
        kw.update(run_kw)
        if self.P is not None:
            kw.setdefault("guess_name", "previous geometry")
            r = self.rhf.run(P0=self.P, **kw)
        else:
            r = self.rhf.run(**kw)
        self.P = r.P
        return r


def scf_at_geometries(mol: Molecule, xyz_list: Sequence[np.ndarray], P0: Optional[torch.Tensor] = None,
                      schwarz_cutoff: float = 1e-12, device: int = 0, **run_kw) -> List[SCFResult]:
    """Converged RHF of ``mol`` at every geometry of ``xyz_list`` (bohr), advanced
    together in one batched context; P0 (a density of ``mol`` in its basis, e.g.
    the last HAR cycle's) seeds every SCF, else each starts from its core guess."""
    mols = [dataclasses.replace(mol, xyz=np.asarray(x, dtype=np.float64).reshape(mol.n_atom, 3))
            for x in xyz_list]
    brhf = BatchRHF(mols, schwarz_cutoff=schwarz_cutoff, device=device)
    starts = None if P0 is None else [P0 for _ in mols]
    try:
        return brhf.run(P0=starts, **run_kw)
    finally:
        brhf.fb.close()
