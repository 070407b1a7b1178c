"""Many RHF SCFs advanced together, one batched J/K build per cycle.

Every cycle issues a single build of a batched context (tf_ctx_create_batch):
each molecule contributes its full density (first cycle, periodic rebuilds and
the final cycles), its density change since the last cycle (incremental
cycles; G is linear in the density), or nothing once converged (a zero change
is screened out entirely by the density test).  Diagonalisations are batched over
molecules of equal size.  Per molecule the loop is Tonto's usual_SCF with DIIS
(keep 8), as in ``tonto_b200.scf``: cheap builds until the convergence test first
passes, then full FP64 builds until it passes again after at least two of them.
A molecule whose DIIS error after ``fallback_after`` cycles is not below its first
cycle's restarts (once) from ``fallback(i)``, as in ``tonto_b200.scf``.
"""

from __future__ import annotations

import time
from typing import Callable, List, Optional

import numpy as np
import torch

from .basis import Molecule
from .fock import TF_JK_DELTA, TF_JK_FULL, TF_JK_MIXED, BatchFockBuilder
from .scf import DIIS, SCFResult


class BatchRHF:
    def __init__(self, mols: List[Molecule], schwarz_cutoff: float = 1e-12, device: int = 0,
                 mixed_fp32_cut: float = 1e-6):
        self.mols = list(mols)
        self.dev = torch.device("cuda", device)
        self.fb = BatchFockBuilder(self.mols, schwarz_cutoff=schwarz_cutoff, device=device,
                                   mixed_fp32_cut=mixed_fp32_cut)
        S, T, V = self.fb.one_electron()
        t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=self.dev)  # noqa: E731
        self.S = [t(x) for x in S]
        self.H = [t(a) + t(b) for a, b in zip(T, V)]
        self.X = []
        for s in self.S:
            e, U = torch.linalg.eigh(s)
            self.X.append((U / torch.sqrt(e)) @ U.T)
        self.n_occ = [m.n_electrons // 2 for m in self.mols]
        self.e_nuc = [m.nuclear_repulsion() for m in self.mols]
        self.off = [int(v) for v in self.fb.offsets]
        tot = self.off[-1]
        self.Xin = torch.zeros(tot, dtype=torch.float64, device=self.dev)
        self.J = torch.zeros(tot, dtype=torch.float64, device=self.dev)
        self.K = torch.zeros(tot, dtype=torch.float64, device=self.dev)
        # molecules grouped by size for batched diagonalisation
        self.by_size = {}
        for i, m in enumerate(self.mols):
            self.by_size.setdefault(m.n_bf, []).append(i)

    def _view(self, buf, i):
        n = self.mols[i].n_bf
        return buf[self.off[i]:self.off[i + 1]].view(n, n)

    def densities(self, Fs, idx):
        """New densities of molecules idx from their (extrapolated) Fock matrices."""
        out = {}
        groups = {}
        for i in idx:
            groups.setdefault(self.mols[i].n_bf, []).append(i)
        for n, ids in groups.items():
            Xs = torch.stack([self.X[i] for i in ids])
            Fo = torch.stack([Fs[i] for i in ids])
            _, C = torch.linalg.eigh(Xs.transpose(1, 2) @ Fo @ Xs)
            C = Xs @ C
            for k, i in enumerate(ids):
                Co = C[k, :, : self.n_occ[i]]
                out[i] = 2.0 * Co @ Co.T
        return out

    def run(self, P0: Optional[List[torch.Tensor]] = None, conv: float = 1e-9, diis_tol: float = 1e-6,
            max_iter: int = 100, incremental: bool = True, mixed: bool = False, rebuild_every: int = 16,
            mixed_until: float = 1e-6, fp64_final: int = 2,
            fallback: Optional[Callable[[int], torch.Tensor]] = None, fallback_after: int = 3) -> List[SCFResult]:
        nm = len(self.mols)
        torch.cuda.synchronize(self.dev)
        t0 = time.perf_counter()
        if P0 is None:
            P = self.densities(self.H, range(nm))
        else:
            P = {i: P0[i].to(self.dev, torch.float64) for i in range(nm)}
        diis = [DIIS(8) for _ in range(nm)]
        F_prev = [None] * nm
        P_prev = [None] * nm
        E_old = [None] * nm
        state = ["cheap" if (incremental or mixed) else "final"] * nm
        n_final = [0] * nm
        since_full = [0] * nm
        done = [False] * nm
        fell_back = [False] * nm
        err_first = [None] * nm
        cyc = [0] * nm
        hist = [[] for _ in range(nm)]
        E = [float("nan")] * nm
        it = 0
        builds = 0
        while not all(done) and it <= max_iter:
            active = [i for i in range(nm) if not done[i]]
            any_final = any(state[i] == "final" for i in active)
            use_mixed = mixed and not any_final and all(
                E_old[i] is None or abs(hist[i][-1][2]) >= mixed_until for i in active)
            kinds = {}
            self.Xin.zero_()
            for i in active:
                delta = (state[i] == "cheap" and incremental and F_prev[i] is not None
                         and since_full[i] < rebuild_every)
                kinds[i] = delta
                self._view(self.Xin, i).copy_(P[i] - P_prev[i] if delta else P[i])
            flags = (TF_JK_MIXED if use_mixed else TF_JK_FULL) | TF_JK_DELTA
            self.fb.make_r_JK_device(self.Xin, self.J, self.K, flags)
            builds += 1
            Fs = {}
            errs = {}
            for i in active:
                J, K = self._view(self.J, i).T, self._view(self.K, i).T     # column-major blocks
                G = J - 0.5 * K
                if kinds[i]:
                    F = F_prev[i] + G
                    since_full[i] += 1
                else:
                    F = self.H[i] + G
                    since_full[i] = 0
                    if state[i] == "final":
                        n_final[i] += 1
                Fs[i] = F
                errs[i] = F @ P[i] @ self.S[i] - self.S[i] @ P[i] @ F
            # scalars of all active molecules in one transfer
            scal = torch.stack([torch.stack([0.5 * torch.sum(P[i] * (self.H[i] + Fs[i])), torch.linalg.norm(errs[i])])
                                for i in active]).cpu().numpy()
            nxt = []
            for k, i in enumerate(active):
                E[i] = float(scal[k, 0]) + self.e_nuc[i]
                err_n = float(scal[k, 1])
                dE = float("inf") if E_old[i] is None else E[i] - E_old[i]
                hist[i].append((it, E[i], dE, err_n, ("mixed" if use_mixed else "fp64") + ("+delta" if kinds[i] else "")))
                if err_first[i] is None:
                    err_first[i] = err_n
                if (fallback is not None and not fell_back[i] and cyc[i] == fallback_after
                        and err_n >= err_first[i]):
                    P[i] = fallback(i).to(self.dev, torch.float64)
                    diis[i].reset()
                    fell_back[i] = True
                    E_old[i] = F_prev[i] = P_prev[i] = err_first[i] = None
                    cyc[i] = 0
                    continue
                cyc[i] += 1
                passed = E_old[i] is not None and abs(dE) < conv and err_n < diis_tol
                if state[i] == "final" and passed and n_final[i] >= min(fp64_final, it + 1):
                    done[i] = True
                    continue
                if state[i] == "cheap" and passed:
                    state[i] = "final"
                E_old[i] = E[i]
                F_prev[i], P_prev[i] = Fs[i], P[i]
                Fs[i] = diis[i].extrapolate(Fs[i], errs[i])
                nxt.append(i)
            if nxt:
                P.update(self.densities(Fs, nxt))
            it += 1
        torch.cuda.synchronize(self.dev)
        secs = time.perf_counter() - t0
        return [SCFResult(energy=E[i], converged=done[i], iterations=len(hist[i]) - 1, builds=builds,
                          seconds=secs, build_seconds=0.0, P=P[i], history=hist[i], fell_back=fell_back[i])
                for i in range(nm)]
