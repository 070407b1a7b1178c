"""Restricted Hartree-Fock SCF driver on the GPU around the J/K builder.

Host-side mirror of Tonto's ``MOLECULE.SCF:usual_SCF`` (molecule.scf.foo:1690-1727):

    initialize_SCF   overlap, core Hamiltonian, initial density (core guess,
                     make_core_mx_guess_MOs :4723, or a caller-supplied one)
    loop             extrapolate_Fock_mx (DIIS on the commutator FPS - SPF, keep 8,
                     :6717-6890) -> update_MOs (diagonalise in the S^-1/2 basis,
                     MO_r_eigen_update :3797) -> make_SCF_density_mx
                     (molecule.base.foo:318) -> make_scf_Fock_mx (:1562, the J/K
                     build through the C ABI) -> energy and convergence
                     (scf_data.foo:2283-2310: |delta E| and the DIIS error both below
                     their tolerances)

The J/K build runs on the device arrays (``tf_build_jk_device``); diagonalisation
and DIIS use torch (cuSOLVER) on the same GPU and stream, so nothing returns to
the host except two scalars per cycle.

Optional modes (none changes the converged answer):
* ``mixed``: quartets below the Schwarz x density cut in FP32 (FP64 roots,
  weights and accumulation); the last ``fp64_final`` cycles rebuilt in FP64;
* ``incremental``: Fock builds from the density change (F_n = F_{n-1} + G[dP]),
  with a full rebuild every ``rebuild_every`` cycles and in the final cycles.
"""

from __future__ import annotations

import dataclasses

import time
from dataclasses import dataclass, field
from typing import Callable, List, Optional

import numpy as np
import torch

from .basis import Molecule
from .fock import TF_JK_DELTA, TF_JK_FULL, TF_JK_MIXED, FockBuilder


def _sync(dev: torch.device) -> None:
    if dev.type == "cuda":
        torch.cuda.synchronize(dev)


@dataclass
class SCFResult:
    energy: float
    converged: bool
    iterations: int
    builds: int
    seconds: float
    build_seconds: float
    P: torch.Tensor
    history: List[tuple] = field(default_factory=list)
    guess: str = "core"
    fell_back: bool = False


class DIIS:
    """Pulay DIIS on the commutator error (Tonto's DIIS, keep 8)."""

    def __init__(self, keep: int = 8):
        self.keep = keep
        self.F: List[torch.Tensor] = []
        self.E: List[torch.Tensor] = []

    def reset(self):
        self.F.clear()
        self.E.clear()

    def extrapolate(self, F: torch.Tensor, err: torch.Tensor) -> torch.Tensor:
        self.F.append(F.clone())
        self.E.append(err.clone())
        if len(self.F) > self.keep:
            self.F.pop(0)
            self.E.pop(0)
        m = len(self.F)
        if m < 2:
            return F
        Es = torch.stack([e.reshape(-1) for e in self.E])
        B = torch.zeros((m + 1, m + 1), dtype=F.dtype, device=F.device)
        B[:m, :m] = Es @ Es.T
        B[m, :m] = -1.0
        B[:m, m] = -1.0
        rhs = torch.zeros(m + 1, dtype=F.dtype, device=F.device)
        rhs[m] = -1.0
        c = torch.linalg.solve(B, rhs)[:m]
        return torch.einsum("i,ijk->jk", c, torch.stack(self.F))


class RHF:
    def __init__(self, mol: Molecule, schwarz_cutoff: float = 1e-12, device: int = 0, diis_keep: int = 8,
                 mixed_fp32_cut: float = 1e-6, builder: Optional[FockBuilder] = None):
        self.mol = mol
        self.dev = device if isinstance(device, torch.device) else torch.device("cuda", device)
        self.fb = builder or FockBuilder(mol, schwarz_cutoff=schwarz_cutoff, device=device,
                                         mixed_fp32_cut=mixed_fp32_cut)
        self._one_electron()
        self.n_occ = mol.n_electrons // 2
        self.diis_keep = diis_keep
        n = mol.n_bf
        self._J = torch.empty((n, n), dtype=torch.float64, device=self.dev)
        self._K = torch.empty((n, n), dtype=torch.float64, device=self.dev)

    def _one_electron(self):
        S, T, V = self.fb.one_electron()
        self.S = torch.tensor(np.ascontiguousarray(S), dtype=torch.float64, device=self.dev)
        self.T = torch.tensor(np.ascontiguousarray(T), dtype=torch.float64, device=self.dev)
        self.V = torch.tensor(np.ascontiguousarray(V), dtype=torch.float64, device=self.dev)
        self.H = self.T + self.V
        e, U = torch.linalg.eigh(self.S)
        self.X = (U / torch.sqrt(e)) @ U.T
        self.e_nuc = self.mol.nuclear_repulsion()

    def set_geometry(self, xyz_bohr) -> None:
        """Move the atoms (same atoms and basis), as Tonto's Hirshfeld-atom refinement
        does between SCFs (molecule.har.foo:352-491): the library rebuilds the pair
        data and Schwarz bounds (tf_set_geometry), the one-electron matrices are
        recomputed, and the next run may start from the previous density."""
        xyz = np.asarray(xyz_bohr, dtype=np.float64).reshape(self.mol.n_atom, 3)
        self.mol = dataclasses.replace(self.mol, xyz=xyz)
        self.fb.set_geometry(xyz)
        self.fb.mol = self.mol
        self._one_electron()

    def density(self, F: torch.Tensor):
        e, C = torch.linalg.eigh(self.X.T @ F @ self.X)
        C = self.X @ C
        Co = C[:, : self.n_occ]
        return 2.0 * Co @ Co.T, e, C

    def core_guess(self) -> torch.Tensor:
        return self.density(self.H)[0]

    def jk(self, P: torch.Tensor, flags: int = TF_JK_FULL):
        Pc = P.contiguous()
        self.fb.make_r_JK_device(Pc, self._J, self._K, flags)
        return self._J, self._K

    def run(self, P0: Optional[torch.Tensor] = None, conv: float = 1e-9, diis_tol: float = 1e-6,
            max_iter: int = 100, mixed: bool = False, fp64_final: int = 2, incremental: bool = False,
            rebuild_every: int = 16, guess_name: str = "core", mixed_until: float = 1e-6,
            fallback: Optional[Callable[[], torch.Tensor]] = None, fallback_after: int = 3,
            loosen: Optional[float] = None, loose_max: float = 1e-10, final_at: float = 10.0,
            verbose: bool = False) -> SCFResult:
        """Converge from P0 (default: core guess).

        With ``mixed`` or ``incremental`` the SCF runs in two states.  "cheap": Fock
        builds from the density change (incremental, a full rebuild every
        ``rebuild_every`` cycles) and, while |dE| >= ``mixed_until``, with FP32
        quartets below the Schwarz x density cut.  Once the DIIS error in the cheap
        state is below ``final_at`` x ``diis_tol`` (or the convergence test passes), the
        SCF continues with full FP64 builds and stops when the test passes after at
        least ``fp64_final`` of them, so the reported energy comes from full FP64 Fock
        matrices; with ``final_at`` > 1 those full builds fall on cycles the SCF needs
        anyway instead of being added after convergence.

        ``fallback``: a callable giving a replacement density; used (once) if the DIIS
        error after ``fallback_after`` cycles is not below the first cycle's.

        ``loosen``: in the cheap state, the Schwarz x density cutoff of each build is
        ``loosen`` times the previous DIIS error, clamped to [the context's cutoff,
        ``loose_max``] (``loose_max`` for the first build), so the bound tightens as the
        SCF converges while the Fock error it admits stays far below the current error;
        the final full FP64 builds always use the context's own cutoff, so the result
        does not depend on it.  With a builder that takes per-molecule cutoffs the cutoff
        is set that way (a device value that a replayed graph build reads, so changing it
        every cycle costs no graph re-capture).
        """
        _sync(self.dev)
        t0 = time.perf_counter()
        tight = self.fb.options.eri_schwarz_cutoff
        per_mol = loosen is not None and hasattr(self.fb, "set_molecule_cutoffs")
        P = self.core_guess() if P0 is None else P0.to(self.dev, torch.float64).contiguous()
        diis = DIIS(self.diis_keep)
        hist = []
        builds = 0
        build_s = 0.0
        E_old = None
        F_prev = P_prev = None
        fell_back = False
        err_first = None
        it = 0
        converged = False
        state = "cheap" if (mixed or incremental) else "final"
        n_final = 0
        since_full = 0
        E = float("nan")
        while True:
            if state == "cheap":
                use_mixed = mixed and not (E_old is not None and abs(hist[-1][2]) < mixed_until)
                use_delta = incremental and F_prev is not None and since_full < rebuild_every
            else:
                use_mixed = use_delta = False
            flags = TF_JK_MIXED if use_mixed else TF_JK_FULL
            if loosen is not None:
                cut = tight
                if state == "cheap" and hist:
                    cut = min(loose_max, max(tight, loosen * hist[-1][3]))
                elif state == "cheap":
                    cut = loose_max
                if per_mol:
                    self.fb.set_molecule_cutoffs([cut])
                elif cut != self.fb.options.eri_schwarz_cutoff:
                    self.fb.set_schwarz_cutoff(cut)
            tb = time.perf_counter()
            if use_delta:
                J, K = self.jk((P - P_prev).contiguous(), flags | TF_JK_DELTA)
                F = F_prev + J - 0.5 * K
                since_full += 1
            else:
                J, K = self.jk(P, flags)
                F = self.H + J - 0.5 * K
                since_full = 0
            kind = ("mixed" if use_mixed else "fp64") + ("+delta" if use_delta else "")
            builds += 1
            if state == "final":
                n_final += 1
            E_t = 0.5 * torch.sum(P * (self.H + F)) + self.e_nuc
            err = F @ P @ self.S - self.S @ P @ F
            err_n_t = torch.linalg.norm(err)
            E, err_n = float(E_t), float(err_n_t)            # the per-cycle host sync
            build_s += time.perf_counter() - tb
            dE = float("inf") if E_old is None else E - E_old
            hist.append((it, E, dE, err_n, kind))
            if verbose:
                print(f"scf {it:3d} E={E:.12f} dE={dE:.3e} err={err_n:.3e} {kind}")
            if err_first is None:
                err_first = err_n
            if fallback is not None and not fell_back and it == fallback_after and err_n >= err_first:
                P = fallback().to(self.dev, torch.float64).contiguous()
                diis.reset()
                fell_back = True
                E_old = None
                F_prev = P_prev = None
                err_first = None
                it += 1
                continue
            passed = E_old is not None and abs(dE) < conv and err_n < diis_tol
            if state == "final" and passed and n_final >= min(fp64_final, it + 1):
                converged = True
                break
            if state == "cheap" and (passed or (E_old is not None and err_n < final_at * diis_tol)):
                state = "final"
            if it >= max_iter:
                break
            E_old = E
            F_prev, P_prev = F, P
            Fx = diis.extrapolate(F, err)
            P, _, _ = self.density(Fx)
            it += 1
        if per_mol:
            self.fb.set_molecule_cutoffs(None)
        if self.fb.options.eri_schwarz_cutoff != tight:
            self.fb.set_schwarz_cutoff(tight)
        _sync(self.dev)
        return SCFResult(energy=E, converged=converged, iterations=it, builds=builds,
                         seconds=time.perf_counter() - t0, build_seconds=build_s, P=P, history=hist,
                         guess=guess_name, fell_back=fell_back)


class UHF(RHF):
    """Unrestricted Hartree-Fock on the unrestricted J/K build (make_u_JK_direct):
    F_a = H + Ja + Jb - Ka, F_b = H + Ja + Jb - Kb; DIIS (keep 8) on both spins
    together, with the commutator errors of both spins as one vector."""

    def __init__(self, mol: Molecule, multiplicity: int = 1, **kw):
        super().__init__(mol, **kw)
        n_el = mol.n_electrons
        n_unp = multiplicity - 1
        if n_unp < 0 or (n_el - n_unp) % 2 or n_unp > n_el:
            raise ValueError("multiplicity does not fit the electron count")
        self.n_alpha = (n_el + n_unp) // 2
        self.n_beta = (n_el - n_unp) // 2
        n = mol.n_bf
        self._buf = [torch.empty((n, n), dtype=torch.float64, device=self.dev) for _ in range(4)]

    def spin_density(self, F: torch.Tensor, n: int) -> torch.Tensor:
        e, C = torch.linalg.eigh(self.X.T @ F @ self.X)
        Co = (self.X @ C)[:, :n]
        return Co @ Co.T

    def run(self, conv: float = 1e-9, diis_tol: float = 1e-6, max_iter: int = 200, flags: int = TF_JK_FULL,
            verbose: bool = False) -> SCFResult:
        _sync(self.dev)
        t0 = time.perf_counter()
        Pa = self.spin_density(self.H, self.n_alpha)
        Pb = self.spin_density(self.H, self.n_beta)
        diis = DIIS(self.diis_keep)
        Ja, Jb, Ka, Kb = self._buf
        E_old = None
        hist = []
        it = 0
        converged = False
        E = float("nan")
        n = self.mol.n_bf
        while True:
            self.fb.make_u_JK_device(Pa.contiguous(), Pb.contiguous(), Ja, Jb, Ka, Kb, flags)
            Fa = self.H + Ja + Jb - Ka
            Fb = self.H + Ja + Jb - Kb
            E = float(0.5 * (torch.sum(Pa * (self.H + Fa)) + torch.sum(Pb * (self.H + Fb)))) + self.e_nuc
            err = torch.cat([Fa @ Pa @ self.S - self.S @ Pa @ Fa, Fb @ Pb @ self.S - self.S @ Pb @ Fb])
            err_n = float(torch.linalg.norm(err))
            dE = float("inf") if E_old is None else E - E_old
            hist.append((it, E, dE, err_n, "fp64"))
            if verbose:
                print(f"uhf {it:3d} E={E:.12f} dE={dE:.3e} err={err_n:.3e}")
            if E_old is not None and abs(dE) < conv and err_n < diis_tol:
                converged = True
                break
            if it >= max_iter:
                break
            E_old = E
            Fx = diis.extrapolate(torch.cat([Fa, Fb]), err)
            Pa = self.spin_density(Fx[:n], self.n_alpha)
            Pb = self.spin_density(Fx[n:], self.n_beta)
            it += 1
        _sync(self.dev)
        res = SCFResult(energy=E, converged=converged, iterations=it, builds=it + 1,
                        seconds=time.perf_counter() - t0, build_seconds=0.0, P=Pa + Pb, history=hist)
        res.Pa, res.Pb = Pa, Pb
        return res
