"""Learned initial density for water clusters.

A 3-layer MLP (width 128, SiLU, FP32 weights) maps a descriptor of each water
pair (v, w) — v == w included — to the density block P(v, w) expressed in the
local frames of v (rows) and w (columns) (``tonto_b200.guess``).  Self blocks are
predicted as corrections to the isolated-water density; pairs with O-O distance
below ``PAIR_CUTOFF`` get a predicted block, farther pairs zero.  The blocks are
rotated to the lab frame and assembled into a full density, which only seeds the
SCF: the converged answer comes from the plain Fock builds, so the network can
change the iteration count but not the result.  If the DIIS error does not fall
within the first cycles, the SCF restarts from the plain guess.

Descriptor (51 values, angstrom, in v's local frame):
    [0]      1 for a self pair, else 0
    [1:10]   O, H1, H2 of w                         (zeros for a self pair)
    [10]     fc(r_vw), fc(r) = (cos(pi r / 6 A) + 1) / 2 for r < 6 A
    [11:51]  the 4 waters nearest to the pair centre (O of v for a self pair,
             the O-O midpoint otherwise), excluding v and w: O, H1, H2 and fc(r)

Training and inference run through the CUDA kernels of include/tontofock_guess.h
(``tf_mlp_*``); torch only holds the device arrays.
"""

from __future__ import annotations

import ctypes
import math
import os
from typing import List, Optional, Tuple

import numpy as np

from .basis import ANGSTROM_PER_BOHR, Molecule
from . import guess as G

PAIR_CUTOFF = 5.0          # angstrom, O-O
ENV_K = 4
RC = 6.0
D_IN = 1 + 9 + 1 + ENV_K * 10
WIDTH = 128
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_WEIGHTS = os.path.join(DATA_DIR, "guess_mlp.npz")


def fc(r: float) -> float:
    return 0.5 * (math.cos(math.pi * r / RC) + 1.0) if r < RC else 0.0


# ---------------------------------------------------------------------------
# descriptors and targets
# ---------------------------------------------------------------------------
def cluster_geometry(mol: Molecule):
    ws, frames, A = G.cluster_rotations(mol)
    xyz = mol.xyz * ANGSTROM_PER_BOHR
    atoms = np.array([[xyz[o], xyz[h1], xyz[h2]] for (o, h1, h2) in ws])      # (n, 3, 3) angstrom
    return ws, frames, A, atoms


def pair_list(atoms: np.ndarray) -> List[Tuple[int, int]]:
    """Every water with itself, then the pairs (v < w) whose O atoms are closer than
    PAIR_CUTOFF, in row order."""
    n = len(atoms)
    out = [(v, v) for v in range(n)]
    if n > 1:
        O = atoms[:, 0]
        d = np.linalg.norm(O[None, :, :] - O[:, None, :], axis=2)
        vs, ws = np.nonzero(np.triu(d < PAIR_CUTOFF, k=1))
        out.extend(zip(vs.tolist(), ws.tolist()))
    return out


def d_in(env_k: int) -> int:
    return 1 + 9 + 1 + env_k * 10


def _fc(r: np.ndarray) -> np.ndarray:
    return np.where(r < RC, 0.5 * (np.cos(np.pi * r / RC) + 1.0), 0.0)


def descriptors(atoms: np.ndarray, frames, pairs, env_k: int = ENV_K) -> np.ndarray:
    """Per pair (v, w), in the local frame R_v of water v with O_v at the origin:
    [v == w], the three atoms of w and fc(|O_w - O_v|) (v != w), then the env_k
    waters u != v, w nearest to the pair centre (O_v, or the O-O midpoint; ties by
    index) with their three atoms and fc(distance to the centre); missing
    neighbours stay zero.  All pairs of a cluster at once."""
    n = len(atoms)
    X = np.zeros((len(pairs), d_in(env_k)), dtype=np.float64)
    if not pairs:
        return X
    P = len(pairs)
    pv = np.array([p[0] for p in pairs])
    pw = np.array([p[1] for p in pairs])
    Rv = np.asarray(frames, dtype=np.float64)[pv]                    # (P, 3, 3), rows = local axes
    O = atoms[:, 0]
    Ov = O[pv]
    same = pv == pw
    diff = ~same

    def local(u):                                                    # (atoms[u] - O_v) @ R_v^T, flattened
        return np.einsum("pak,pjk->paj", atoms[u] - Ov[:, None, :], Rv).reshape(P, 9)

    X[same, 0] = 1.0
    X[diff, 1:10] = local(pw)[diff]
    X[diff, 10] = _fc(np.linalg.norm(O[pw] - Ov, axis=1))[diff]
    centre = np.where(same[:, None], Ov, 0.5 * (Ov + O[pw]))
    dist = np.linalg.norm(O[None, :, :] - centre[:, None, :], axis=2)  # (P, n)
    masked = dist.copy()
    rows = np.arange(P)
    masked[rows, pv] = np.inf
    masked[rows, pw] = np.inf
    order = np.argsort(masked, axis=1, kind="stable")
    n_others = n - np.where(same, 1, 2)
    for j in range(min(env_k, n)):
        ok = j < n_others
        u = order[:, j]
        base = 11 + 10 * j
        X[ok, base:base + 9] = local(u)[ok]
        X[ok, base + 9] = _fc(dist[rows, u])[ok]
    return X


def local_blocks(mol: Molecule, P: np.ndarray, A, pairs, P_mono_local: np.ndarray) -> np.ndarray:
    rng = G.water_ao_ranges(mol)
    m = P_mono_local.shape[0]
    Y = np.zeros((len(pairs), m * m))
    for k, (v, w) in enumerate(pairs):
        (a0, a1), (b0, b1) = rng[v], rng[w]
        B = G.to_local(P[a0:a1, b0:b1], A[v], A[w])
        if v == w:
            B = B - P_mono_local
        Y[k] = B.ravel()
    return Y


def assemble(mol: Molecule, A, pairs, Y: np.ndarray, P_mono_local: np.ndarray) -> np.ndarray:
    rng = G.water_ao_ranges(mol)
    m = P_mono_local.shape[0]
    P = np.zeros((mol.n_bf, mol.n_bf))
    for k, (v, w) in enumerate(pairs):
        B = Y[k].reshape(m, m)
        (a0, a1), (b0, b1) = rng[v], rng[w]
        if v == w:
            B = 0.5 * (B + B.T) + P_mono_local
            P[a0:a1, a0:a1] = A[v].T @ B @ A[v]
        else:
            blk = A[v].T @ B @ A[w]
            P[a0:a1, b0:b1] = blk
            P[b0:b1, a0:a1] = blk.T
    return P


# ---------------------------------------------------------------------------
# the network, on the CUDA kernels
# ---------------------------------------------------------------------------
def _lib():
    from .fock import load_library
    L = load_library()
    if not getattr(L, "_mlp_bound", False):
        vp, i, f, lg = ctypes.c_void_p, ctypes.c_int, ctypes.c_float, ctypes.c_long
        L.tf_mlp_gemm.argtypes = [i, i, i, vp, lg, lg, vp, lg, lg, vp, i, vp, vp, f, vp]
        L.tf_mlp_silu_bwd.argtypes = [lg, vp, vp, vp, vp]
        L.tf_mlp_colsum.argtypes = [i, i, vp, vp, vp]
        L.tf_mlp_mse.argtypes = [i, i, vp, vp, vp, f, vp, vp, i, vp]
        L.tf_mlp_adam.argtypes = [lg, vp, vp, vp, vp, f, f, f, f, i, f, vp]
        L._mlp_bound = True
    return L


def _p(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _ck(rc):
    if rc != 0:
        raise RuntimeError(f"tf_mlp kernel error {rc}")


class MLP:
    """x -> SiLU(W1 x + b1) -> SiLU(W2 . + b2) -> W3 . + b3, FP32 on the GPU."""

    def __init__(self, d_in: int, d_out: int, width: int = WIDTH, device: int = 0, seed: int = 0):
        import torch
        self.torch = torch
        self.dev = torch.device("cuda", device)
        g = np.random.default_rng(seed)
        shapes = [(width, d_in), (width,), (width, width), (width,), (d_out, width), (d_out,)]
        self.params = []
        for s in shapes:
            if len(s) == 2:
                w = g.normal(size=s) * math.sqrt(2.0 / s[1])
            else:
                w = np.zeros(s)
            self.params.append(torch.tensor(w, dtype=torch.float32, device=self.dev))
        self.grads = [torch.zeros_like(p) for p in self.params]
        self.m = [torch.zeros_like(p) for p in self.params]
        self.v = [torch.zeros_like(p) for p in self.params]
        self.step_count = 0
        self.d_in, self.d_out, self.width = d_in, d_out, width
        self.env_k = (d_in - 11) // 10            # environment waters in the descriptor
        self.x_mean = np.zeros(d_in)
        self.x_std = np.ones(d_in)
        self.y_mean = np.zeros(d_out)
        self.y_std = np.ones(d_out)

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def forward(self, X, keep: bool = False):
        """X: (B, d_in) float32 CUDA tensor (normalised).  Returns Y (B, d_out)."""
        torch = self.torch
        L = _lib()
        W1, b1, W2, b2, W3, b3 = self.params
        B = X.shape[0]
        s = self._stream()
        Z1 = torch.empty((B, self.width), dtype=torch.float32, device=self.dev)
        A1 = torch.empty_like(Z1)
        Z2 = torch.empty_like(Z1)
        A2 = torch.empty_like(Z1)
        Y = torch.empty((B, self.d_out), dtype=torch.float32, device=self.dev)
        # Z = X W^T + b: A(i,k) = X[i*d_in + k], B(k,j) = W[j*d_in + k]
        _ck(L.tf_mlp_gemm(B, self.width, self.d_in, _p(X), self.d_in, 1, _p(W1), 1, self.d_in, _p(b1), 1, _p(Z1),
                          _p(A1), 0.0, s))
        _ck(L.tf_mlp_gemm(B, self.width, self.width, _p(A1), self.width, 1, _p(W2), 1, self.width, _p(b2), 1,
                          _p(Z2), _p(A2), 0.0, s))
        _ck(L.tf_mlp_gemm(B, self.d_out, self.width, _p(A2), self.width, 1, _p(W3), 1, self.width, _p(b3), 0, None,
                          _p(Y), 0.0, s))
        if keep:
            self._cache = (X, Z1, A1, Z2, A2)
        return Y

    def backward(self, dY):
        """Gradients of the parameters for the upstream gradient dY (B, d_out)."""
        torch = self.torch
        L = _lib()
        X, Z1, A1, Z2, A2 = self._cache
        W1, b1, W2, b2, W3, b3 = self.params
        gW1, gb1, gW2, gb2, gW3, gb3 = self.grads
        B = X.shape[0]
        s = self._stream()
        w, d_in, d_out = self.width, self.d_in, self.d_out
        # dW3 = dY^T A2: A(i,k) = dY[k*d_out + i], B(k,j) = A2[k*w + j]
        _ck(L.tf_mlp_gemm(d_out, w, B, _p(dY), 1, d_out, _p(A2), w, 1, None, 0, None, _p(gW3), 0.0, s))
        _ck(L.tf_mlp_colsum(B, d_out, _p(dY), _p(gb3), s))
        dA2 = torch.empty_like(A2)
        # dA2 = dY W3: A(i,k) = dY[i*d_out + k], B(k,j) = W3[k*w + j]
        _ck(L.tf_mlp_gemm(B, w, d_out, _p(dY), d_out, 1, _p(W3), w, 1, None, 0, None, _p(dA2), 0.0, s))
        dZ2 = torch.empty_like(Z2)
        _ck(L.tf_mlp_silu_bwd(B * w, _p(dA2), _p(Z2), _p(dZ2), s))
        _ck(L.tf_mlp_gemm(w, w, B, _p(dZ2), 1, w, _p(A1), w, 1, None, 0, None, _p(gW2), 0.0, s))
        _ck(L.tf_mlp_colsum(B, w, _p(dZ2), _p(gb2), s))
        dA1 = torch.empty_like(A1)
        _ck(L.tf_mlp_gemm(B, w, w, _p(dZ2), w, 1, _p(W2), w, 1, None, 0, None, _p(dA1), 0.0, s))
        dZ1 = torch.empty_like(Z1)
        _ck(L.tf_mlp_silu_bwd(B * w, _p(dA1), _p(Z1), _p(dZ1), s))
        _ck(L.tf_mlp_gemm(w, d_in, B, _p(dZ1), 1, w, _p(X), d_in, 1, None, 0, None, _p(gW1), 0.0, s))
        _ck(L.tf_mlp_colsum(B, w, _p(dZ1), _p(gb1), s))
        return self.grads

    def mse(self, Y, T, weights=None):
        """Mean squared error over all elements (weighted per row) and dY."""
        torch = self.torch
        L = _lib()
        B, N = Y.shape
        dY = torch.empty_like(Y)
        nb = 256
        part = torch.zeros(nb, dtype=torch.float32, device=self.dev)
        _ck(L.tf_mlp_mse(B, N, _p(Y), _p(T), _p(weights), 1.0 / (B * N), _p(dY), _p(part), nb, self._stream()))
        return part.sum(), dY

    def adam(self, lr: float, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        L = _lib()
        self.step_count += 1
        s = self._stream()
        for p, g, m, v in zip(self.params, self.grads, self.m, self.v):
            _ck(L.tf_mlp_adam(p.numel(), _p(p), _p(g), _p(m), _p(v), lr, beta1, beta2, eps, self.step_count,
                              weight_decay, s))

    def predict(self, X_raw: np.ndarray) -> np.ndarray:
        torch = self.torch
        Xn = ((X_raw - self.x_mean) / self.x_std).astype(np.float32)
        Y = self.forward(torch.tensor(Xn, device=self.dev))
        return Y.cpu().numpy().astype(np.float64) * self.y_std + self.y_mean

    def save(self, path: str, extra: Optional[dict] = None):
        d = {f"p{i}": p.cpu().numpy() for i, p in enumerate(self.params)}
        d.update(x_mean=self.x_mean, x_std=self.x_std, y_mean=self.y_mean, y_std=self.y_std,
                 dims=np.array([self.d_in, self.d_out, self.width]))
        if extra:
            d.update(extra)
        np.savez_compressed(path, **d)

    @classmethod
    def load(cls, path: str = DEFAULT_WEIGHTS, device: int = 0) -> "MLP":
        import torch
        z = np.load(path)
        d_in, d_out, width = (int(v) for v in z["dims"])
        m = cls(d_in, d_out, width, device=device)
        for i in range(6):
            m.params[i] = torch.tensor(z[f"p{i}"], dtype=torch.float32, device=m.dev)
        m.x_mean, m.x_std, m.y_mean, m.y_std = z["x_mean"], z["x_std"], z["y_mean"], z["y_std"]
        m.extra = {k: z[k] for k in z.files if k.startswith("mono") or k.startswith("meta")}
        return m


def learned_density(mol: Molecule, model: MLP, P_mono_local: np.ndarray) -> np.ndarray:
    """Initial density of a water cluster from the network."""
    ws, frames, A, atoms = cluster_geometry(mol)
    pairs = pair_list(atoms)
    X = descriptors(atoms, frames, pairs, model.env_k)
    Y = model.predict(X)
    return assemble(mol, A, pairs, Y, P_mono_local)


def learned_densities(mols: List[Molecule], model: MLP, P_mono_local: np.ndarray) -> List[np.ndarray]:
    """Initial densities of many clusters, one network evaluation over all their pairs."""
    geo = [cluster_geometry(m) for m in mols]
    pairs = [pair_list(g[3]) for g in geo]
    X = np.concatenate([descriptors(g[3], g[1], p, model.env_k) for g, p in zip(geo, pairs)])
    Y = model.predict(X)
    out, k = [], 0
    for m, g, p in zip(mols, geo, pairs):
        out.append(assemble(m, g[2], p, Y[k:k + len(p)], P_mono_local))
        k += len(p)
    return out
