"""Many RHF SCFs advanced together, one batched J/K build per cycle.

Every cycle issues a single build of a batched context (tf_ctx_create_batch):
each molecule contributes its full density (first cycle, periodic rebuilds and
the final cycles), its density change since the last cycle (incremental
cycles; G is linear in the density), or nothing once converged (a zero change
is screened out entirely by the density test).  Per molecule the loop is Tonto's
usual_SCF with DIIS (keep 8), as in ``tonto_b200.scf``: cheap builds until the
DIIS error is within ``final_at`` times its tolerance (or the convergence test
passes), then full FP64 builds until the test passes after at least two of them.  A molecule whose DIIS error after ``fallback_after`` cycles
is not below its first cycle's restarts (once) from ``fallback(i)``.

Everything between the builds runs on the device in batches: the molecules are
grouped into a few size buckets, each padded to its largest member, and the
Fock matrices, energies, DIIS errors, DIIS extrapolations and new densities of a
bucket are batched matrix products.  The density of an (extrapolated) Fock matrix
is the projector on its n_occ lowest orbitals; it is obtained by trace-correcting
purification (Niklasson, Phys. Rev. B 66, 155115 (2002), "TC2") of the Fock
matrix in the orthogonal basis: X_0 = (e_max - F') / (e_max - e_min) with
Gershgorin bounds, then X <- X^2 or 2X - X^2, whichever moves tr X towards
n_occ, until X is idempotent.  This is the same projector as the aufbau density
from a diagonalisation (the SCF converges to the same fixed point), at the cost
of batched matrix products instead of one eigensolver call per molecule.
"""

from __future__ import annotations

import time
from typing import Callable, List, Optional

import numpy as np
import torch

from .basis import Molecule
from .fock import TF_JK_DELTA, TF_JK_FULL, TF_JK_MIXED, BatchFockBuilder
from .scf import SCFResult, _sync


class _Bucket:
    """Molecules of similar size, padded to the largest (n)."""

    def __init__(self, ids: List[int], n_bf: List[int], dev):
        self.ids = ids
        self.m = len(ids)
        self.n = max(n_bf[i] for i in ids)
        self.n_bf = torch.tensor([n_bf[i] for i in ids], device=dev)
        r = torch.arange(self.n, device=dev)
        self.valid = r[None, :] < self.n_bf[:, None]                       # (m, n) real rows


def purify(Fo: torch.Tensor, valid: torch.Tensor, n_occ: torch.Tensor, tol: float = 1e-13,
           max_iter: int = 100) -> torch.Tensor:
    """TC2 purification of a batch of symmetric matrices Fo (m, n, n) (orthogonal
    basis; rows with valid == False are padding): the projector on the n_occ[i]
    lowest eigenvectors of each real block (padding stays unoccupied)."""
    m, n, _ = Fo.shape
    eye = torch.eye(n, dtype=Fo.dtype, device=Fo.device)
    Fo = Fo * (valid[:, :, None] & valid[:, None, :])
    d = torch.diagonal(Fo, dim1=1, dim2=2)
    r = Fo.abs().sum(2) - d.abs()
    big = torch.finfo(Fo.dtype).max
    e_min = torch.where(valid, d - r, torch.full_like(d, big)).min(1).values
    e_max = torch.where(valid, d + r, torch.full_like(d, -big)).max(1).values
    # padding rows get e_max on the diagonal: they map to 0 and stay there
    Fo = Fo + torch.diag_embed((~valid).to(Fo.dtype) * e_max[:, None])
    X = (e_max[:, None, None] * eye - Fo) / (e_max - e_min)[:, None, None]
    N = n_occ.to(Fo.dtype)
    for it in range(max_iter):
        X2 = torch.bmm(X, X)
        t1 = torch.diagonal(X, dim1=1, dim2=2).sum(1)
        t2 = torch.diagonal(X2, dim1=1, dim2=2).sum(1)
        square = (t2 - N).abs() < (2.0 * t1 - t2 - N).abs()
        X = torch.where(square[:, None, None], X2, 2.0 * X - X2)
        if it >= 8 and it % 4 == 0 and float((t1 - t2).abs().max()) < tol * n:   # tr(X - X^2)
            break
    return 0.5 * (X + X.transpose(1, 2))


class BatchRHF:
    def __init__(self, mols: List[Molecule], schwarz_cutoff: float = 1e-12, device: int = 0,
                 mixed_fp32_cut: float = 1e-6, n_buckets: int = 4, builder=None):
        self.mols = list(mols)
        nm = len(self.mols)
        self.dev = device if isinstance(device, torch.device) else torch.device("cuda", device)
        dev = self.dev
        self.fb = builder or BatchFockBuilder(self.mols, schwarz_cutoff=schwarz_cutoff, device=device,
                                              mixed_fp32_cut=mixed_fp32_cut)
        n_bf = [m.n_bf for m in self.mols]
        self.n_bf = n_bf
        order = sorted(range(nm), key=lambda i: n_bf[i])
        nb = max(1, min(n_buckets, nm))
        cuts = [order[(k * nm) // nb:((k + 1) * nm) // nb] for k in range(nb)]
        self.buckets = [_Bucket(ids, n_bf, dev) for ids in cuts if ids]
        # concatenated <-> padded index maps (the matrices are symmetric)
        self.off = [int(v) for v in self.fb.offsets]
        for b in self.buckets:                    # built on the device
            idx = []
            for k, i in enumerate(b.ids):
                r = torch.arange(n_bf[i], device=dev)
                idx.append((k * b.n * b.n + r[:, None] * b.n + r[None, :]).reshape(-1))
            b.pad_idx = torch.cat(idx)
            b.cat_idx = torch.cat([torch.arange(self.off[i], self.off[i + 1], device=dev) for i in b.ids])
        S, T, V = self.fb.one_electron()
        for b in self.buckets:
            b.S = self._pad(b, [S[i] for i in b.ids])
            b.H = self._pad(b, [T[i] + V[i] for i in b.ids])
            # orthogonaliser X = L^-T from the Cholesky factor S = L L^T (padding: identity):
            # X^T S X = 1, and the densities do not depend on which orthogonaliser is used
            pad_eye = torch.diag_embed((~b.valid).to(torch.float64))
            L = torch.linalg.cholesky(b.S + pad_eye)
            eye = torch.eye(b.n, dtype=torch.float64, device=dev).expand(b.m, b.n, b.n)
            b.X = torch.linalg.solve_triangular(L, eye, upper=False).transpose(1, 2).contiguous()
            b.n_occ = torch.tensor([self.mols[i].n_electrons // 2 for i in b.ids], device=dev)
            b.e_nuc = torch.tensor([self.mols[i].nuclear_repulsion() for i in b.ids], dtype=torch.float64,
                                   device=dev)
        tot = self.off[-1]
        self.Xin = torch.zeros(tot, dtype=torch.float64, device=dev)
        self.J = torch.zeros(tot, dtype=torch.float64, device=dev)
        self.K = torch.zeros(tot, dtype=torch.float64, device=dev)

    def _pad(self, b: _Bucket, mats) -> torch.Tensor:
        out = torch.zeros((b.m, b.n, b.n), dtype=torch.float64, device=self.dev)
        for k, a in enumerate(mats):
            n = a.shape[0]
            out[k, :n, :n] = torch.as_tensor(np.ascontiguousarray(a) if isinstance(a, np.ndarray) else a,
                                             dtype=torch.float64, device=self.dev)
        return out

    def _from_cat(self, b: _Bucket, buf: torch.Tensor) -> torch.Tensor:
        out = torch.zeros(b.m * b.n * b.n, dtype=torch.float64, device=self.dev)
        out[b.pad_idx] = buf[b.cat_idx]
        return out.view(b.m, b.n, b.n)

    def _to_cat(self, b: _Bucket, X: torch.Tensor, buf: torch.Tensor):
        buf[b.cat_idx] = X.reshape(-1)[b.pad_idx]

    def densities(self, b: _Bucket, F: torch.Tensor) -> torch.Tensor:
        """Aufbau densities 2 C_occ C_occ^T of a bucket's Fock matrices (padded)."""
        Fo = torch.bmm(b.X.transpose(1, 2), torch.bmm(F, b.X))
        Po = purify(Fo, b.valid, b.n_occ)
        return 2.0 * torch.bmm(b.X, torch.bmm(Po, b.X.transpose(1, 2)))

    def run(self, P0: Optional[List[torch.Tensor]] = None, conv: float = 1e-9, diis_tol: float = 1e-6,
            max_iter: int = 100, incremental: bool = True, mixed: bool = False, rebuild_every: int = 16,
            mixed_until: float = 1e-6, fp64_final: int = 2, final_at: float = 10.0,
            fallback: Optional[Callable[[int], torch.Tensor]] = None, fallback_after: int = 3,
            diis_keep: int = 8, loosen: Optional[float] = None, loose_max: float = 1e-10) -> List[SCFResult]:
        nm = len(self.mols)
        dev = self.dev
        _sync(dev)
        t0 = time.perf_counter()
        tight = self.fb.options.eri_schwarz_cutoff
        per_mol = loosen is not None and hasattr(self.fb, "set_molecule_cutoffs")
        bk = self.buckets
        for b in bk:
            if P0 is None:
                b.P = self.densities(b, b.H)
            else:
                b.P = self._pad(b, [P0[i].to(dev, torch.float64) for i in b.ids])
            b.P_prev = torch.zeros_like(b.P)
            b.F_prev = torch.zeros_like(b.P)
            b.Fh = torch.zeros((b.m, diis_keep) + b.P.shape[1:], dtype=torch.float64, device=dev)
            b.Eh = torch.zeros_like(b.Fh)
            b.count = torch.zeros(b.m, dtype=torch.long, device=dev)
        where, row = {}, {}
        r0 = 0
        for bi, b in enumerate(bk):
            for k, i in enumerate(b.ids):
                where[i] = (bi, k)
                row[i] = r0 + k
            r0 += b.m
        E_old = [None] * nm
        state = ["cheap" if (incremental or mixed) else "final"] * nm
        n_final = [0] * nm
        since_full = [0] * nm
        done = [False] * nm
        fell_back = [False] * nm
        err_first = [None] * nm
        cyc = [0] * nm
        have_prev = [False] * nm
        hist = [[] for _ in range(nm)]
        E = [float("nan")] * nm
        it = 0
        builds = 0
        mask = lambda b, v: torch.tensor([v[i] for i in b.ids], device=dev)  # noqa: E731
        while not all(done) and it <= max_iter:
            active = [i for i in range(nm) if not done[i]]
            any_final = any(state[i] == "final" for i in active)
            use_mixed = mixed and not any_final and all(
                E_old[i] is None or abs(hist[i][-1][2]) >= mixed_until for i in active)
            delta = [(not done[i]) and state[i] == "cheap" and incremental and have_prev[i]
                     and since_full[i] < rebuild_every for i in range(nm)]
            live = [not d for d in done]
            for b in bk:
                dm = mask(b, delta)[:, None, None]
                D = torch.where(dm, b.P - b.P_prev, b.P) * mask(b, live)[:, None, None]
                self._to_cat(b, D, self.Xin)
            flags = (TF_JK_MIXED if use_mixed else TF_JK_FULL) | TF_JK_DELTA
            if loosen is not None:
                # cheap cycles: a Schwarz x density cutoff that follows the DIIS error
                # (the Fock error it admits stays far below it), loose_max before the
                # first error is known; the context's own cutoff for the final full FP64
                # builds, whose Fock matrices are then exact.  Per molecule when the
                # builder takes per-molecule cutoffs, else one cutoff for the build: the
                # least error of the active molecules, the tight one once any is final.
                def cheap_cut(i):
                    return loose_max if not hist[i] else min(loose_max, max(tight, loosen * hist[i][-1][3]))
                if per_mol:
                    self.fb.set_molecule_cutoffs([tight if (done[i] or state[i] == "final") else cheap_cut(i)
                                                  for i in range(nm)])
                else:
                    cut = tight if any_final else min(cheap_cut(i) for i in active)
                    if cut != self.fb.options.eri_schwarz_cutoff:
                        self.fb.set_schwarz_cutoff(cut)
            self.fb.make_r_JK_device(self.Xin, self.J, self.K, flags)
            builds += 1
            scal = []
            for b in bk:
                G = self._from_cat(b, self.J) - 0.5 * self._from_cat(b, self.K)
                b.F = torch.where(mask(b, delta)[:, None, None], b.F_prev + G, b.H + G)
                b.err = torch.bmm(b.F, torch.bmm(b.P, b.S)) - torch.bmm(b.S, torch.bmm(b.P, b.F))
                e_b = 0.5 * (b.P * (b.H + b.F)).sum((1, 2)) + b.e_nuc
                scal.append(torch.stack([e_b, torch.linalg.norm(b.err.reshape(b.m, -1), dim=1)], 1))
            scal = torch.cat(scal).cpu().numpy()                 # the per-cycle host sync
            cont = [False] * nm
            restart = []
            for i in active:
                E[i] = float(scal[row[i], 0])
                err_n = float(scal[row[i], 1])
                dE = float("inf") if E_old[i] is None else E[i] - E_old[i]
                hist[i].append((it, E[i], dE, err_n, ("mixed" if use_mixed else "fp64") + ("+delta" if delta[i] else "")))
                if delta[i]:
                    since_full[i] += 1
                else:
                    since_full[i] = 0
                    if state[i] == "final":
                        n_final[i] += 1
                if err_first[i] is None:
                    err_first[i] = err_n
                if (fallback is not None and not fell_back[i] and cyc[i] == fallback_after
                        and err_n >= err_first[i]):
                    restart.append(i)
                    fell_back[i] = True
                    E_old[i] = err_first[i] = None
                    have_prev[i] = False
                    cyc[i] = 0
                    continue
                cyc[i] += 1
                passed = E_old[i] is not None and abs(dE) < conv and err_n < diis_tol
                if state[i] == "final" and passed and n_final[i] >= min(fp64_final, it + 1):
                    done[i] = True
                    continue
                if state[i] == "cheap" and (passed or (E_old[i] is not None and err_n < final_at * diis_tol)):
                    state[i] = "final"
                E_old[i] = E[i]
                have_prev[i] = True
                cont[i] = True
            # DIIS (keep 8) and new densities of the molecules that go on
            for b in bk:
                cm = mask(b, cont)
                if not any(cont[i] for i in b.ids):
                    continue
                c3 = cm[:, None, None]
                b.P_prev = torch.where(c3, b.P, b.P_prev)
                b.F_prev = torch.where(c3, b.F, b.F_prev)
                Fx = self._diis(b, cm, diis_keep)
                b.P = torch.where(c3, self.densities(b, Fx), b.P)
            for i in restart:
                bi, k = where[i]
                b = bk[bi]
                n = self.n_bf[i]
                b.P[k].zero_()
                b.P[k, :n, :n] = fallback(i).to(dev, torch.float64)
                b.count[k] = 0
            it += 1
        if per_mol:
            self.fb.set_molecule_cutoffs(None)
        if self.fb.options.eri_schwarz_cutoff != tight:
            self.fb.set_schwarz_cutoff(tight)
        _sync(dev)
        secs = time.perf_counter() - t0
        out = []
        for i in range(nm):
            bi, k = where[i]
            n = self.n_bf[i]
            out.append(SCFResult(energy=E[i], converged=done[i], iterations=len(hist[i]) - 1, builds=builds,
                                 seconds=secs, build_seconds=0.0, P=bk[bi].P[k, :n, :n].clone(),
                                 history=hist[i], fell_back=fell_back[i]))
        return out

    @staticmethod
    def _diis(b: _Bucket, cm: torch.Tensor, keep: int) -> torch.Tensor:
        """Pulay DIIS per molecule of a bucket; the rows cm store this cycle's F and
        commutator error first (a ring of the last ``keep``)."""
        dev = b.F.device
        pos = b.count % keep
        sel = torch.arange(b.m, device=dev)[cm]
        b.Fh[sel, pos[cm]] = b.F[cm]
        b.Eh[sel, pos[cm]] = b.err[cm]
        b.count = torch.where(cm, b.count + 1, b.count)
        used = torch.arange(keep, device=dev)[None, :] < b.count.clamp(max=keep)[:, None]      # (m, keep)
        Ef = b.Eh.reshape(b.m, keep, -1)
        B = torch.bmm(Ef, Ef.transpose(1, 2))
        scale = torch.diagonal(B, dim1=1, dim2=2).amax(1).clamp(min=1e-300)
        B = B / scale[:, None, None]
        um = used[:, :, None] & used[:, None, :]
        eye = torch.eye(keep, dtype=B.dtype, device=dev)
        B = torch.where(um, B, eye.expand_as(B) * (~used)[:, :, None].to(B.dtype))
        A = torch.zeros((b.m, keep + 1, keep + 1), dtype=B.dtype, device=dev)
        A[:, :keep, :keep] = B
        A[:, :keep, keep] = -used.to(B.dtype)
        A[:, keep, :keep] = -used.to(B.dtype)
        A[:, keep, keep] = (b.count == 0).to(B.dtype)      # nothing stored yet: keeps the system regular
        rhs = torch.zeros((b.m, keep + 1), dtype=B.dtype, device=dev)
        rhs[:, keep] = -1.0
        c = torch.linalg.solve(A, rhs)[:, :keep]
        Fx = torch.einsum("mk,mkij->mij", c, b.Fh)
        return torch.where((b.count < 2)[:, None, None], b.F, Fx)
