"""CPU ORACLE — test infrastructure only.

ctypes front end to ``libtonto_oracle.so`` (the C++ restatement of Tonto's
restricted direct J/K build in ``tonto_oracle.cpp``) plus a numpy restatement of
Tonto's RHF SCF loop (molecule.scf.foo:1690-1727 usual_SCF; core guess
molecule.scf.foo:4723; DIIS extrapolation molecule.scf.foo:6717-6890 with the
commutator error FPS - SPF; convergence scf_data.foo:2283-2310 requires both
|delta E| and the DIIS error below their tolerances).

Only ``tests/``, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg use
this module, and only as the checker.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import time
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtonto_oracle.so")

_lib = None


def build() -> str:
    """Compile the oracle library (make, system g++ with OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.c_int, dp, ctypes.c_int, ip, ip, ip, ip, dp, dp, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_max_I.argtypes = [ctypes.c_void_p, dp]
        L.oracle_shell_quartet.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, dp]
        L.oracle_shell_quartet.restype = ctypes.c_int
        L.oracle_jk.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_long, ctypes.c_int]
        L.oracle_jk_sample.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_long, ctypes.c_int, ctypes.c_long,
                                       ctypes.c_long]
        L.oracle_counts.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
        L.oracle_flops.argtypes = [ctypes.c_void_p, dp, ctypes.c_int]
        L.oracle_last_times.argtypes = [ctypes.c_void_p, dp]
        L.oracle_fp32_bound.argtypes = [ctypes.c_void_p, dp, ctypes.c_double, dp, dp]
        L.oracle_fp32_bound.restype = ctypes.c_long
        L.oracle_jk_quartets.argtypes = [ctypes.c_void_p, dp, dp, dp, ctypes.c_long, ip, ip, ctypes.c_int]
        L.oracle_jk_uhf.argtypes = [ctypes.c_void_p, dp, dp, dp, dp, dp, dp, ctypes.c_int]
        L.oracle_spherical_matrix.argtypes = [ctypes.c_int, dp]
        L.oracle_spherical_matrix.restype = ctypes.c_int
        L.oracle_components.argtypes = [ctypes.c_int, ip]
        L.oracle_components.restype = ctypes.c_int
        L.oracle_rys.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.oracle_one_electron.argtypes = [ctypes.c_void_p, dp, dp, dp, dp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class Oracle:
    """The reference J/K build for one molecule (positions fixed at creation)."""

    def __init__(self, mol, schwarz_cutoff: float = 1e-12, pair_cutoff: float = 1e-6):
        self.mol = mol
        sa, sl, sn, sf, ex, co = mol.flat_arrays()
        self._keep = [np.ascontiguousarray(mol.xyz, dtype=np.float64), sa, sl, sn, sf, ex, co]
        xyz = self._keep[0]
        self.n_bf = mol.n_bf
        self.n_pairs = mol.n_shell * (mol.n_shell + 1) // 2
        self.h = lib().oracle_create(mol.n_atom, _dp(xyz), mol.n_shell, _ip(sa), _ip(sl), _ip(sn), _ip(sf),
                                     _dp(ex), _dp(co), int(mol.spherical), schwarz_cutoff, pair_cutoff)

    def __del__(self):
        h = getattr(self, "h", None)
        if h and lib is not None:            # (module globals may be gone at interpreter exit)
            lib().oracle_destroy(h)
            self.h = None

    def max_I(self) -> np.ndarray:
        out = np.zeros(self.n_pairs)
        lib().oracle_max_I(self.h, _dp(out))
        return out

    def shell_quartet(self, a: int, b: int, c: int, d: int, skip: bool = False) -> np.ndarray:
        m = self.mol
        dims = [m.shell_nbf(m.shells[s].l) for s in (a, b, c, d)]
        out = np.zeros(int(np.prod(dims)))
        lib().oracle_shell_quartet(self.h, a, b, c, d, int(skip), _dp(out))
        return out.reshape(dims[::-1]).transpose(3, 2, 1, 0)   # (a,b,c,d)

    def jk(self, P: np.ndarray, max_ab_pairs: int = -1, n_threads: int = 0):
        """J, K (Tonto's make_r_JK_direct) for density P (symmetric, n_bf x n_bf)."""
        Pf = np.asfortranarray(P, dtype=np.float64)
        J = np.zeros((self.n_bf, self.n_bf), order="F")
        K = np.zeros((self.n_bf, self.n_bf), order="F")
        lib().oracle_jk(self.h, _dp(Pf), _dp(J), _dp(K), int(max_ab_pairs), int(n_threads))
        return np.ascontiguousarray(J), np.ascontiguousarray(K)

    def jk_sample(self, P: np.ndarray, stride: int, offset: int = 0, n_threads: int = 0) -> float:
        """Time the outer loop over ab = offset, offset+stride, ... (seconds, whole call)."""
        Pf = np.asfortranarray(P, dtype=np.float64)
        J = np.zeros((self.n_bf, self.n_bf), order="F")
        K = np.zeros((self.n_bf, self.n_bf), order="F")
        t = time.perf_counter()
        lib().oracle_jk_sample(self.h, _dp(Pf), _dp(J), _dp(K), -1, int(n_threads), int(stride), int(offset))
        return time.perf_counter() - t

    def jk_sample_times(self, P: np.ndarray, stride: int, offset: int = 0, n_threads: int = 0):
        """(loop seconds, whole-call seconds) of the bra pairs ab = offset, offset+stride, ...:
        the shell-quartet loop of that share alone, and the call with its fixed work (density
        maxima, per-thread accumulators, their sum, fold and reflect), which one full build
        does once whatever the share."""
        Pf = np.asfortranarray(P, dtype=np.float64)
        J = np.zeros((self.n_bf, self.n_bf), order="F")
        K = np.zeros((self.n_bf, self.n_bf), order="F")
        lib().oracle_jk_sample(self.h, _dp(Pf), _dp(J), _dp(K), -1, int(n_threads), int(stride), int(offset))
        return self.last_times()

    def last_times(self):
        out = np.zeros(2)
        lib().oracle_last_times(self.h, _dp(out))
        return float(out[0]), float(out[1])

    def flops(self, reset: bool = False) -> np.ndarray:
        """Counted FLOPs of the J/K calls so far, shape (5, 5, 5, 5, 8): per (la lb|lc ld)
        class, the categories set-up, pair terms, roots, recurrences, (e0|f0) sums,
        transfers, spherical transform, digestion."""
        out = np.zeros(625 * 8)
        lib().oracle_flops(self.h, _dp(out), int(reset))
        return out.reshape(5, 5, 5, 5, 8)

    def jk_shard(self, P: np.ndarray, rank: int, n_ranks: int, n_threads: int = 0):
        """Partial J, K of the bra pairs ab = rank, rank + n_ranks, ... (one rank of
        Tonto's round-robin parallel do); the ranks' results sum to jk(P)."""
        Pf = np.asfortranarray(P, dtype=np.float64)
        J = np.zeros((self.n_bf, self.n_bf), order="F")
        K = np.zeros((self.n_bf, self.n_bf), order="F")
        lib().oracle_jk_sample(self.h, _dp(Pf), _dp(J), _dp(K), -1, int(n_threads), int(n_ranks), int(rank))
        return np.ascontiguousarray(J), np.ascontiguousarray(K)

    def jk_quartets(self, P: np.ndarray, bra: np.ndarray, ket: np.ndarray, n_threads: int = 0):
        """J, K of the shell quartets (bra[i] | ket[i]) (Tonto pair indices, either order)
        with make_r_JK_direct's screening, factors, digestion and fold."""
        Pf = np.asfortranarray(P, dtype=np.float64)
        bra = np.ascontiguousarray(bra, dtype=np.int32)
        ket = np.ascontiguousarray(ket, dtype=np.int32)
        J = np.zeros((self.n_bf, self.n_bf), order="F")
        K = np.zeros((self.n_bf, self.n_bf), order="F")
        lib().oracle_jk_quartets(self.h, _dp(Pf), _dp(J), _dp(K), len(bra), _ip(bra), _ip(ket), int(n_threads))
        return np.ascontiguousarray(J), np.ascontiguousarray(K)

    def fp32_bound(self, P: np.ndarray, fp32_cut: float):
        """(Jb, Kb, n): per element, the sum of the term bounds a mixed-precision build
        evaluates in FP32 (quartets passing the screen with bound below fp32_cut), and
        their number.  An FP32 evaluation with relative error delta is within delta Jb,
        delta Kb of the FP64 build."""
        Pf = np.asfortranarray(P, dtype=np.float64)
        Jb = np.zeros((self.n_bf, self.n_bf), order="F")
        Kb = np.zeros((self.n_bf, self.n_bf), order="F")
        n = lib().oracle_fp32_bound(self.h, _dp(Pf), float(fp32_cut), _dp(Jb), _dp(Kb))
        return np.ascontiguousarray(Jb), np.ascontiguousarray(Kb), int(n)

    def jk_uhf(self, Pa: np.ndarray, Pb: np.ndarray, n_threads: int = 0):
        """Unrestricted (Ja, Jb, Ka, Kb) (Tonto's make_u_JK_direct): screened on Pa + Pb."""
        Pa = np.asfortranarray(Pa, dtype=np.float64)
        Pb = np.asfortranarray(Pb, dtype=np.float64)
        out = [np.zeros((self.n_bf, self.n_bf), order="F") for _ in range(4)]
        lib().oracle_jk_uhf(self.h, _dp(Pa), _dp(Pb), *[_dp(x) for x in out], int(n_threads))
        return tuple(np.ascontiguousarray(x) for x in out)

    FLOP_CATEGORIES = ("setup", "pair", "roots", "vrr", "form", "hrr", "spherical", "digest")

    def counts(self, reset: bool = False) -> np.ndarray:
        """Contracted and primitive quartets computed so far, shape (5, 5, 5, 5, 2).
        reset clears these and the FLOP counters."""
        out = np.zeros(625 * 2)
        lib().oracle_counts(self.h, _dp(out), int(reset))
        return out.reshape(5, 5, 5, 5, 2)

    def one_electron(self):
        S = np.zeros((self.n_bf, self.n_bf), order="F")
        T = np.zeros_like(S)
        V = np.zeros_like(S)
        Z = np.ascontiguousarray(self.mol.Z, dtype=np.float64)
        lib().oracle_one_electron(self.h, _dp(Z), _dp(S), _dp(T), _dp(V))
        return np.ascontiguousarray(S), np.ascontiguousarray(T), np.ascontiguousarray(V)


def spherical_matrix(l: int) -> np.ndarray:
    n = (l + 1) * (l + 2) // 2
    out = np.zeros(n * (2 * l + 1))
    lib().oracle_spherical_matrix(l, _dp(out))
    return out.reshape(n, 2 * l + 1)


def components(l: int) -> np.ndarray:
    n = (l + 1) * (l + 2) // 2
    out = np.zeros(3 * n, dtype=np.int32)
    lib().oracle_components(l, _ip(out))
    return out.reshape(n, 3)


def rys(n: int, x: float):
    u = np.zeros(n)
    w = np.zeros(n)
    lib().oracle_rys(n, float(x), _dp(u), _dp(w))
    return u, w


# ---------------------------------------------------------------------------
# RHF SCF (restatement of usual_SCF with core guess and DIIS)
# ---------------------------------------------------------------------------

def orthogonaliser(S: np.ndarray) -> np.ndarray:
    e, U = np.linalg.eigh(S)
    return (U / np.sqrt(e)) @ U.T


def density_from_fock(F: np.ndarray, X: np.ndarray, n_occ: int):
    e, C = np.linalg.eigh(X.T @ F @ X)
    C = X @ C
    Co = C[:, :n_occ]
    return 2.0 * Co @ Co.T, e, C


class DIIS:
    def __init__(self, keep: int = 8):
        self.keep = keep
        self.F = []
        self.E = []

    def extrapolate(self, F: np.ndarray, err: np.ndarray) -> np.ndarray:
        self.F.append(F.copy())
        self.E.append(err.copy())
        if len(self.F) > self.keep:
            self.F.pop(0)
            self.E.pop(0)
        m = len(self.F)
        if m < 2:
            return F
        B = np.zeros((m + 1, m + 1))
        for i in range(m):
            for j in range(i + 1):
                B[i, j] = B[j, i] = float(np.vdot(self.E[i], self.E[j]))
        B[m, :m] = B[:m, m] = -1.0
        rhs = np.zeros(m + 1)
        rhs[m] = -1.0
        try:
            c = np.linalg.solve(B, rhs)[:m]
        except np.linalg.LinAlgError:
            return F
        return sum(ci * Fi for ci, Fi in zip(c, self.F))


def scf(mol, orc: Optional[Oracle] = None, P0: Optional[np.ndarray] = None, conv: float = 1e-9,
        diis_tol: float = 1e-6, diis_keep: int = 8, max_iter: int = 100, verbose: bool = False) -> Dict:
    """Converged RHF with the oracle's J/K.  Returns energies, density, iterations."""
    orc = orc or Oracle(mol)
    S, T, V = orc.one_electron()
    H = T + V
    X = orthogonaliser(S)
    n_occ = mol.n_electrons // 2
    enuc = mol.nuclear_repulsion()
    t0 = time.time()
    if P0 is None:
        P, _, _ = density_from_fock(H, X, n_occ)
    else:
        P = P0.copy()
    diis = DIIS(diis_keep)
    E_old = None
    it = 0
    n_builds = 0
    err_norm = np.inf
    history = []
    while True:
        J, K = orc.jk(P)
        n_builds += 1
        F = H + J - 0.5 * K
        E = 0.5 * float(np.sum(P * (H + F))) + enuc
        err = F @ P @ S - S @ P @ F
        err_norm = float(np.linalg.norm(err))
        dE = np.inf if E_old is None else E - E_old
        history.append((it, E, dE, err_norm))
        if verbose:
            print(f"oracle scf {it:3d} E={E:.12f} dE={dE:.3e} err={err_norm:.3e}")
        if E_old is not None and abs(dE) < conv and err_norm < diis_tol:
            break
        if it >= max_iter:
            break
        E_old = E
        Fx = diis.extrapolate(F, err)
        P, eps, C = density_from_fock(Fx, X, n_occ)
        it += 1
    Vee = 0.5 * float(np.sum(P * (J - 0.5 * K)))
    return {"E": E, "E_e": E - enuc, "V_NN": enuc, "V_ee": Vee, "T": float(np.sum(P * T)),
            "V_eN": float(np.sum(P * V)), "P": P, "iterations": it, "builds": n_builds,
            "seconds": time.time() - t0, "history": history, "S": S, "H": H}


def uhf_scf(mol, n_alpha: int, n_beta: int, orc: Optional[Oracle] = None, conv: float = 1e-9,
            diis_tol: float = 1e-6, diis_keep: int = 8, max_iter: int = 200, verbose: bool = False) -> Dict:
    """Converged UHF with the oracle's unrestricted J/K, from the core guess:
    F_a = H + Ja + Jb - Ka, F_b = H + Ja + Jb - Kb, DIIS on both spins together."""
    orc = orc or Oracle(mol)
    S, T, V = orc.one_electron()
    H = T + V
    X = orthogonaliser(S)
    enuc = mol.nuclear_repulsion()
    Pa, _, _ = density_from_fock(H, X, n_alpha)
    Pb, _, _ = density_from_fock(H, X, n_beta)
    Pa, Pb = 0.5 * Pa, 0.5 * Pb          # density_from_fock gives 2 C C^T (closed-shell convention)
    diis = DIIS(diis_keep)
    E_old = None
    it = 0
    history = []
    while True:
        Ja, Jb, Ka, Kb = orc.jk_uhf(Pa, Pb)
        Fa = H + Ja + Jb - Ka
        Fb = H + Ja + Jb - Kb
        E = 0.5 * float(np.sum(Pa * (H + Fa)) + np.sum(Pb * (H + Fb))) + enuc
        ea = Fa @ Pa @ S - S @ Pa @ Fa
        eb = Fb @ Pb @ S - S @ Pb @ Fb
        err = np.concatenate([ea, eb])
        err_norm = float(np.linalg.norm(err))
        dE = np.inf if E_old is None else E - E_old
        history.append((it, E, dE, err_norm))
        if verbose:
            print(f"oracle uhf {it:3d} E={E:.12f} dE={dE:.3e} err={err_norm:.3e}")
        if E_old is not None and abs(dE) < conv and err_norm < diis_tol:
            break
        if it >= max_iter:
            break
        E_old = E
        Fx = diis.extrapolate(np.concatenate([Fa, Fb]), err)
        n = Fa.shape[0]
        Pa = 0.5 * density_from_fock(Fx[:n], X, n_alpha)[0]
        Pb = 0.5 * density_from_fock(Fx[n:], X, n_beta)[0]
        it += 1
    return {"E": E, "Pa": Pa, "Pb": Pb, "iterations": it, "history": history}
