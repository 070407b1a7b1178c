"""Host-side mirror of Tonto's J/K builder interface over the C ABI (include/tontofock.h).

``FockBuilder`` plays the role of ``MOLECULE.FOCK`` for one molecule:

* ``make_r_JK(P)``        -> (J, K)      as make_r_JK_direct / make_r_JK_engine
                                          (molecule.fock.foo:1235-1505)
* ``make_r_Fock_mx(P, H)`` -> F = H + J - K/2  as make_r_Fock_mx (:88-155)
* ``max_I``               -> Schwarz bounds as initialize_max_I (:3705-3752)

Arrays are numpy (host) or torch CUDA tensors (device entry point).  The CUDA
library is required: if it cannot be loaded, or no device is present, the calls
raise — there is no CPU fallback.
"""

from __future__ import annotations

import ctypes
import os
from typing import Optional, Tuple

import numpy as np

from .basis import Molecule

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtontofock.so")

TF_JK_FULL = 0x0
TF_JK_MIXED = 0x1
TF_JK_DELTA = 0x2
TF_JK_J_ONLY = 0x8
TF_JK_K_ONLY = 0x10


class TontoFockError(RuntimeError):
    pass


class _Basis(ctypes.Structure):
    _fields_ = [("n_atom", ctypes.c_int), ("xyz", ctypes.POINTER(ctypes.c_double)),
                ("n_shell", ctypes.c_int), ("shell_atom", ctypes.POINTER(ctypes.c_int)),
                ("shell_l", ctypes.POINTER(ctypes.c_int)), ("shell_nprim", ctypes.POINTER(ctypes.c_int)),
                ("shell_first_bf", ctypes.POINTER(ctypes.c_int)), ("exponents", ctypes.POINTER(ctypes.c_double)),
                ("coefficients", ctypes.POINTER(ctypes.c_double)), ("is_spherical", ctypes.c_int)]


class Options(ctypes.Structure):
    _fields_ = [("eri_schwarz_cutoff", ctypes.c_double), ("eri_primitive_pair_cutoff", ctypes.c_double),
                ("mixed_fp32_cut", ctypes.c_double), ("device", ctypes.c_int), ("deterministic", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("build_ms", ctypes.c_double), ("eri_ms", ctypes.c_double), ("quartets", ctypes.c_double),
                ("quartets_fp32", ctypes.c_double), ("prim_quartets", ctypes.c_double),
                ("flops", ctypes.c_double), ("h2d_bytes", ctypes.c_longlong), ("d2h_bytes", ctypes.c_longlong),
                ("kernels", ctypes.c_int), ("graph", ctypes.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Tune(ctypes.Structure):
    _fields_ = [("streams", ctypes.c_int), ("candidates", ctypes.c_int), ("ms", ctypes.c_double * 8),
                ("direct_ms", ctypes.c_double), ("variant_classes", ctypes.c_int)]

    def as_dict(self):
        return {"streams": self.streams, "candidates": self.candidates, "direct_ms": self.direct_ms,
                "ms": [self.ms[i] for i in range(self.candidates)], "variant_classes": self.variant_classes}


class ClassStats(ctypes.Structure):
    _fields_ = [("l", ctypes.c_int * 4), ("quartets", ctypes.c_double), ("prim_quartets", ctypes.c_double),
                ("flops", ctypes.c_double), ("ms", ctypes.c_double)]


_lib = None


def load_library(path: Optional[str] = None):
    """Load libtontofock.so (built in-tree by tonto_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise TontoFockError(f"CUDA library missing: {path} (run python -m tonto_b200.build)")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    d, i, vp = ctypes.c_double, ctypes.c_int, ctypes.c_void_p
    L.tf_default_options.argtypes = [P(Options)]
    L.tf_ctx_create.argtypes = [P(_Basis), P(Options), P(vp)]
    L.tf_set_geometry.argtypes = [vp, P(d)]
    L.tf_build_jk.argtypes = [vp, P(d), P(d), P(d), i]
    L.tf_set_shard.argtypes = [vp, i, i]
    L.tf_set_schwarz_cutoff.argtypes = [vp, d]
    L.tf_set_molecule_cutoffs.argtypes = [vp, P(d)]
    L.tf_set_list_budget.argtypes = [vp, ctypes.c_longlong]
    L.tf_set_kernel_variant.argtypes = [vp, ctypes.c_int]
    L.tf_set_screen_record_budget.argtypes = [vp, ctypes.c_longlong]
    L.tf_set_graph.argtypes = [vp, i]
    L.tf_build_jk_uhf.argtypes = [vp, P(d), P(d), P(d), P(d), P(d), P(d), i]
    L.tf_build_jk_uhf_device.argtypes = [vp, vp, vp, vp, vp, vp, vp, i, vp]
    L.tf_autotune.argtypes = [vp, vp, vp, vp, i, i, P(Tune)]
    L.tf_build_jk_device.argtypes = [vp, vp, vp, vp, i, vp]
    L.tf_build_fock.argtypes = [vp, P(d), P(d), P(d)]
    L.tf_build_jk_batch.argtypes = [P(vp), i, P(P(d)), P(P(d)), P(P(d)), i]
    L.tf_ctx_create_batch.argtypes = [P(_Basis), i, P(Options), P(vp)]
    L.tf_batch_info.argtypes = [vp, P(i)]
    L.tf_build_jk_batched.argtypes = [vp, P(P(d)), P(P(d)), P(P(d)), i]
    L.tf_one_electron.argtypes = [vp, P(d), P(d), P(d), P(d)]
    L.tf_last_stats.argtypes = [vp, P(Stats)]
    L.tf_last_class_stats.argtypes = [vp, P(ClassStats), i]
    L.tf_n_bf.argtypes = [vp]
    L.tf_schwarz.argtypes = [vp, P(d)]
    L.tf_ctx_destroy.argtypes = [vp]
    L.tf_debug_fail_alloc.argtypes = [i]
    L.tf_plan_shards.argtypes = [P(_Basis), P(d), d, i, P(ctypes.c_longlong), P(i), P(i), P(i), P(i), P(i), P(d)]
    L.tf_build_jk_f.argtypes = [vp, P(d), P(d), P(d), i, P(i)]
    L.tf_build_jk_f.restype = None
    L.tf_build_fock_f.argtypes = [vp, P(d), P(d), P(d), P(i)]
    L.tf_build_fock_f.restype = None
    L.tf_build_jk_uhf_f.argtypes = [vp, P(d), P(d), P(d), P(d), P(d), P(d), i, P(i)]
    L.tf_build_jk_uhf_f.restype = None
    L.tf_error_string.argtypes = [i]
    L.tf_error_string.restype = ctypes.c_char_p
    L.tf_version.restype = ctypes.c_char_p
    _lib = L
    return L


def _check(rc: int):
    if rc != 0:
        raise TontoFockError(f"tontofock error {rc}: {load_library().tf_error_string(rc).decode()}")


def default_options(**kw) -> Options:
    o = Options()
    _check(load_library().tf_default_options(ctypes.byref(o)))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _basis_struct(mol: Molecule, keep: list) -> _Basis:
    sa, sl, sn, sf, ex, co = mol.flat_arrays()
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64)
    keep += [xyz, sa, sl, sn, sf, ex, co]
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))  # noqa: E731
    return _Basis(mol.n_atom, _dp(xyz), mol.n_shell, ip(sa), ip(sl), ip(sn), ip(sf), _dp(ex), _dp(co),
                  int(mol.spherical))


class FockBuilder:
    """Direct J/K builder for one molecule on one GPU (C ABI context)."""

    def __init__(self, mol: Molecule, schwarz_cutoff: float = 1e-9, pair_cutoff: float = 1e-6,
                 device: int = 0, mixed_fp32_cut: float = 1e-6, deterministic: bool = False):
        L = load_library()
        self.mol = mol
        self._arrays = []
        self._basis = _basis_struct(mol, self._arrays)
        self.options = default_options(eri_schwarz_cutoff=schwarz_cutoff, eri_primitive_pair_cutoff=pair_cutoff,
                                       device=device, mixed_fp32_cut=mixed_fp32_cut,
                                       deterministic=int(deterministic))
        h = ctypes.c_void_p()
        _check(L.tf_ctx_create(ctypes.byref(self._basis), ctypes.byref(self.options), ctypes.byref(h)))
        self.h = h
        self.n_bf = L.tf_n_bf(h)

    def close(self):
        if getattr(self, "h", None):
            load_library().tf_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_geometry(self, xyz_bohr: np.ndarray):
        x = np.ascontiguousarray(xyz_bohr, dtype=np.float64)
        _check(load_library().tf_set_geometry(self.h, _dp(x)))

    def set_schwarz_cutoff(self, cutoff: float):
        """Schwarz x density cutoff of the following builds."""
        _check(load_library().tf_set_schwarz_cutoff(self.h, float(cutoff)))
        self.options.eri_schwarz_cutoff = float(cutoff)

    def set_molecule_cutoffs(self, cutoffs):
        """Per-molecule Schwarz x density cutoffs of the following builds (one value per
        molecule of the context, in place of the context's cutoff); None returns every
        molecule to the context's cutoff."""
        L = load_library()
        if cutoffs is None:
            _check(L.tf_set_molecule_cutoffs(self.h, None))
            return
        c = np.ascontiguousarray(cutoffs, dtype=np.float64)
        n = len(getattr(self, "mols", [self.mol]))
        if c.shape != (n,):
            raise ValueError(f"{n} cutoffs expected")
        _check(L.tf_set_molecule_cutoffs(self.h, _dp(c)))

    def set_list_budget(self, quartets: int):
        """Largest quartet-list chunk (entries of 8 bytes) a build keeps on the device."""
        _check(load_library().tf_set_list_budget(self.h, int(quartets)))

    def set_screen_record_budget(self, n_bytes: int):
        """Device bytes for the screening record (0: the list write screens again)."""
        _check(load_library().tf_set_screen_record_budget(self.h, int(n_bytes)))

    def set_kernel_variant(self, variant: int):
        """Run every class pair's kernel in one variant (0 .. 3; see tf_set_kernel_variant)."""
        _check(load_library().tf_set_kernel_variant(self.h, int(variant)))

    def set_graph(self, on: bool):
        """Replay builds as one captured CUDA graph (default) or launch class by class."""
        _check(load_library().tf_set_graph(self.h, int(bool(on))))

    def autotune(self, P, J, K, flags: int = TF_JK_FULL, max_streams: int = 4) -> dict:
        """Choose the class schedule of graph builds by timing (device arrays as make_r_JK_device)."""
        import torch
        for t in (P, J, K):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise ValueError("autotune takes contiguous float64 CUDA arrays")
        res = Tune()
        _check(load_library().tf_autotune(self.h, ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(J.data_ptr()),
                                          ctypes.c_void_p(K.data_ptr()), int(flags), int(max_streams),
                                          ctypes.byref(res)))
        return res.as_dict()

    def set_shard(self, index: int, count: int):
        """Build only shard ``index`` of ``count`` (the bra tasks tf_plan_shards deals to
        it by estimated cost); the shards' J and K sum to the full build."""
        _check(load_library().tf_set_shard(self.h, int(index), int(count)))

    @property
    def max_I(self) -> np.ndarray:
        n = self.mol.n_shell * (self.mol.n_shell + 1) // 2
        out = np.zeros(n)
        _check(load_library().tf_schwarz(self.h, _dp(out)))
        return out

    def make_r_JK(self, P: np.ndarray, flags: int = TF_JK_FULL, out=None) -> Tuple[np.ndarray, np.ndarray]:
        """J, K for the symmetric density P (host arrays; Fortran-ordered results).
        ``out``: a pair of Fortran-contiguous float64 (n_bf, n_bf) arrays to write J and K
        into (for instance views of page-locked buffers, which the copies back reach
        faster), else new arrays."""
        n = self.n_bf
        Pf = np.asfortranarray(P, dtype=np.float64)
        if Pf.shape != (n, n):
            raise ValueError(f"P must be {n}x{n}")
        if out is None:
            J = np.empty((n, n), order="F")
            K = np.empty((n, n), order="F")
        else:
            J, K = out
            for a in (J, K):
                if a.shape != (n, n) or a.dtype != np.float64 or not a.flags.f_contiguous or not a.flags.writeable:
                    raise ValueError(f"out arrays must be writeable Fortran-contiguous float64 {n}x{n}")
        _check(load_library().tf_build_jk(self.h, _dp(Pf), _dp(J), _dp(K), int(flags)))
        return J, K

    def make_r_JK_device(self, P, J, K, flags: int = TF_JK_FULL, stream=None):
        """J, K on device (torch CUDA float64 tensors of shape (n_bf, n_bf) on the context's
        GPU), ordered after the earlier work on ``stream`` (a torch.cuda.Stream, default: the
        current stream) and before its later work; returns when the build has finished."""
        import torch
        for t in (P, J, K):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() == self.n_bf ** 2):
                raise ValueError("device J/K tensors must be contiguous float64 CUDA (n_bf, n_bf)")
            self._on_device(t)
        s = stream if stream is not None else torch.cuda.current_stream(P.device)
        _check(load_library().tf_build_jk_device(self.h, ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(J.data_ptr()),
                                                 ctypes.c_void_p(K.data_ptr()), int(flags),
                                                 ctypes.c_void_p(s.cuda_stream)))

    def make_u_JK(self, Pa: np.ndarray, Pb: np.ndarray, flags: int = TF_JK_FULL):
        """Unrestricted (Ja, Jb, Ka, Kb) from the alpha and beta densities (host arrays):
        MOLECULE.FOCK:make_u_JK_direct."""
        n = self.n_bf
        Pa = np.asfortranarray(Pa, dtype=np.float64)
        Pb = np.asfortranarray(Pb, dtype=np.float64)
        if Pa.shape != (n, n) or Pb.shape != (n, n):
            raise ValueError(f"Pa, Pb must be {n}x{n}")
        out = [np.empty((n, n), order="F") for _ in range(4)]
        _check(load_library().tf_build_jk_uhf(self.h, _dp(Pa), _dp(Pb), *[_dp(x) for x in out], int(flags)))
        return tuple(out)

    def make_u_JK_device(self, Pa, Pb, Ja, Jb, Ka, Kb, flags: int = TF_JK_FULL, stream=None):
        """Unrestricted J, K on device tensors (n_bf, n_bf), ordered on ``stream``."""
        import torch
        for t in (Pa, Pb, Ja, Jb, Ka, Kb):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() == self.n_bf ** 2):
                raise ValueError("device tensors must be contiguous float64 CUDA (n_bf, n_bf)")
            self._on_device(t)
        s = stream if stream is not None else torch.cuda.current_stream(Pa.device)
        ptr = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
        _check(load_library().tf_build_jk_uhf_device(self.h, ptr(Pa), ptr(Pb), ptr(Ja), ptr(Jb), ptr(Ka), ptr(Kb),
                                                     int(flags), ctypes.c_void_p(s.cuda_stream)))

    def make_r_Fock_mx(self, P: np.ndarray, H: np.ndarray) -> np.ndarray:
        """F = H + J - K/2 for the density P and core Hamiltonian H (host arrays):
        MOLECULE.FOCK:make_r_Fock_mx."""
        n = self.n_bf
        Pf = np.asfortranarray(P, dtype=np.float64)
        Hf = np.asfortranarray(H, dtype=np.float64)
        if Pf.shape != (n, n) or Hf.shape != (n, n):
            raise ValueError(f"P and H must be {n}x{n}")
        F = np.empty((n, n), order="F")
        _check(load_library().tf_build_fock(self.h, _dp(Pf), _dp(Hf), _dp(F)))
        return F

    def _on_device(self, t):
        if t.device.index != self.options.device:
            raise ValueError(f"tensor on {t.device}, context on cuda:{self.options.device}")

    def class_stats(self) -> list:
        """Per-class (la lb|lc ld) figures of the last build."""
        L = load_library()
        n = L.tf_last_class_stats(self.h, None, 0)
        arr = (ClassStats * max(n, 1))()
        L.tf_last_class_stats(self.h, arr, n)
        sym = "spdfg"
        out = []
        for c in arr[:n]:
            name = "(%s%s|%s%s)" % tuple(sym[v] for v in c.l)
            out.append({"class": name, "quartets": c.quartets, "prim_quartets": c.prim_quartets,
                        "flops": c.flops, "ms": c.ms})
        return out

    def one_electron(self):
        """S, T, V in the Tonto basis (make_overlap_mx, make_kinetic_energy_mx,
        make_nuclear_attraction_mx)."""
        n = self.n_bf
        Z = np.ascontiguousarray(self.mol.Z, dtype=np.float64)
        S = np.empty((n, n), order="F")
        T = np.empty((n, n), order="F")
        V = np.empty((n, n), order="F")
        _check(load_library().tf_one_electron(self.h, _dp(Z), _dp(S), _dp(T), _dp(V)))
        return S, T, V

    def stats(self) -> dict:
        s = Stats()
        _check(load_library().tf_last_stats(self.h, ctypes.byref(s)))
        return s.as_dict()


class BatchFockBuilder(FockBuilder):
    """J/K builds of many independent molecules in one launch sequence (a batched
    context).  Device arrays hold the molecules' n_bf x n_bf blocks concatenated."""

    def __init__(self, mols, schwarz_cutoff: float = 1e-9, pair_cutoff: float = 1e-6, device: int = 0,
                 mixed_fp32_cut: float = 1e-6, deterministic: bool = False):
        L = load_library()
        self.mols = list(mols)
        self.mol = self.mols[0]
        self._arrays = []
        arr = (_Basis * len(self.mols))(*[_basis_struct(m, self._arrays) for m in self.mols])
        self._basis = arr
        self.options = default_options(eri_schwarz_cutoff=schwarz_cutoff, eri_primitive_pair_cutoff=pair_cutoff,
                                       device=device, mixed_fp32_cut=mixed_fp32_cut,
                                       deterministic=int(deterministic))
        h = ctypes.c_void_p()
        _check(L.tf_ctx_create_batch(arr, len(self.mols), ctypes.byref(self.options), ctypes.byref(h)))
        self.h = h
        nb = (ctypes.c_int * len(self.mols))()
        L.tf_batch_info(h, nb)
        self.n_bf_per_mol = [int(v) for v in nb]
        self.offsets = np.concatenate([[0], np.cumsum([n * n for n in self.n_bf_per_mol])]).astype(np.int64)
        self.n_bf = L.tf_n_bf(h)

    def make_r_JK_batched(self, Ps, flags: int = TF_JK_FULL):
        """J, K per molecule from host densities Ps[i] (n_bf_i x n_bf_i)."""
        n = len(self.mols)
        if len(Ps) != n:
            raise ValueError(f"{n} densities expected")
        Pf = [np.asfortranarray(P, dtype=np.float64) for P in Ps]
        for P, nb in zip(Pf, self.n_bf_per_mol):
            if P.shape != (nb, nb):
                raise ValueError(f"density of shape {P.shape}, molecule has {nb} functions")
        Js = [np.empty_like(p, order="F") for p in Pf]
        Ks = [np.empty_like(p, order="F") for p in Pf]
        arr = lambda lst: (ctypes.POINTER(ctypes.c_double) * n)(*[_dp(a) for a in lst])  # noqa: E731
        _check(load_library().tf_build_jk_batched(self.h, arr(Pf), arr(Js), arr(Ks), int(flags)))
        return Js, Ks

    def make_r_JK_device(self, P, J, K, flags: int = TF_JK_FULL, stream=None):
        """P, J, K: contiguous float64 CUDA tensors of the concatenated blocks."""
        import torch
        tot = int(self.offsets[-1])
        for t in (P, J, K):
            if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous() and t.numel() == tot):
                raise ValueError("batched device arrays must be contiguous float64 CUDA of the concatenated size")
            self._on_device(t)
        s = stream if stream is not None else torch.cuda.current_stream(P.device)
        _check(load_library().tf_build_jk_device(self.h, ctypes.c_void_p(P.data_ptr()), ctypes.c_void_p(J.data_ptr()),
                                                 ctypes.c_void_p(K.data_ptr()), int(flags),
                                                 ctypes.c_void_p(s.cuda_stream)))

    def one_electron(self):
        """S, T, V per molecule (lists)."""
        Z = np.concatenate([np.asarray(m.Z, dtype=np.float64) for m in self.mols])
        tot = int(self.offsets[-1])
        S, T, V = np.empty(tot), np.empty(tot), np.empty(tot)
        _check(load_library().tf_one_electron(self.h, _dp(Z), _dp(S), _dp(T), _dp(V)))
        out = []
        for X in (S, T, V):
            out.append([X[self.offsets[i]:self.offsets[i + 1]].reshape(n, n).T.copy()
                        for i, n in enumerate(self.n_bf_per_mol)])
        return out
