"""The no-allocation one-electron entry point, checked against the allocating one.

tf_one_electron_noalloc serves callers that cannot call cudaMalloc where they need
the integrals (a host framework that owns the GPU memory, or code where an
allocation is forbidden or would stall the device).  It keeps all scratch in one
fixed array in device memory and writes into arrays the caller already owns.  Two
calls in a row, on different molecules, must each match tf_one_electron; so must
two calls queued back to back on one stream with no synchronisation between them,
and a call whose (pinned) host inputs the caller overwrites as soon as it returns.
This file is collected last so that a failure here cannot stop the rest of the
suite.
"""

import ctypes

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster

TOL = 1e-12
TF_EINVAL, TF_EUNSUPPORTED = -1, -4


def _lib():
    from tonto_b200.fock import _Basis, load_library
    L = load_library()
    L.tf_one_electron_noalloc.argtypes = [ctypes.POINTER(_Basis), ctypes.POINTER(ctypes.c_double),
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    return L


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class _Inputs:
    """The host arrays of one call (kept alive with the struct that points at them)."""

    def __init__(self, mol, pinned=False):
        from tonto_b200.fock import _Basis
        sa, sl, sn, sf, ex, co = mol.flat_arrays()
        arrs = [np.ascontiguousarray(mol.xyz, dtype=np.float64), np.ascontiguousarray(mol.Z, dtype=np.float64),
                sa, sl, sn, sf, ex, co]
        if pinned:                                # page-locked copies: the copies to the device are truly async
            import torch
            pin = []
            for a in arrs:
                t = torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.int32).pin_memory()
                v = t.numpy()
                v[...] = a
                pin.append((t, v))
            self._torch = [t for t, _ in pin]
            arrs = [v for _, v in pin]
        self.xyz, self.Z, self.sa, self.sl, self.sn, self.sf, self.ex, self.co = arrs
        self.basis = _Basis(mol.n_atom, _dp(self.xyz), mol.n_shell, _ip(self.sa), _ip(self.sl), _ip(self.sn),
                            _ip(self.sf), _dp(self.ex), _dp(self.co), int(mol.spherical))


def _call(L, inp, outs, stream=None):
    return L.tf_one_electron_noalloc(ctypes.byref(inp.basis), _dp(inp.Z), *[ctypes.c_void_p(t.data_ptr()) for t in outs],
                                     ctypes.c_void_p(stream.cuda_stream) if stream is not None else None)


def _check(outs, mol):
    from tonto_b200.fock import FockBuilder
    fb = FockBuilder(mol)
    ref = fb.one_electron()
    fb.close()
    # outputs are column-major n x n; the matrices are symmetric
    for got, r in zip(outs, ref):
        g = got.cpu().numpy().T
        assert np.all(np.isfinite(g))
        assert np.max(np.abs(g - r)) <= TOL


@pytest.mark.gpu
def test_noalloc_one_electron_matches_allocating_entry_point(cuda_ok):
    import torch
    L = _lib()
    dev = torch.device("cuda", 0)
    for mol in (water_cluster(2, seed=3), water_cluster(3, seed=5, spherical=False)):
        n = mol.n_bf
        inp = _Inputs(mol)
        # caller-owned outputs, filled with garbage so that a missed element shows
        out = [torch.full((n, n), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
        torch.cuda.synchronize(dev)
        rc = _call(L, inp, out)
        assert rc == 0, L.tf_error_string(rc)
        torch.cuda.synchronize(dev)
        _check(out, mol)


@pytest.mark.gpu
def test_noalloc_two_calls_back_to_back_on_one_stream(cuda_ok):
    import torch
    L = _lib()
    dev = torch.device("cuda", 0)
    mols = (water_cluster(3, seed=11), water_cluster(2, seed=12, spherical=False))
    inps = [_Inputs(m) for m in mols]
    outs = [[torch.full((m.n_bf, m.n_bf), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
            for m in mols]
    s = torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    for inp, out in zip(inps, outs):              # no synchronisation between the two calls
        rc = _call(L, inp, out, s)
        assert rc == 0, L.tf_error_string(rc)
    s.synchronize()
    for out, m in zip(outs, mols):
        _check(out, m)


@pytest.mark.gpu
def test_noalloc_pinned_inputs_may_be_overwritten_on_return(cuda_ok):
    import torch
    L = _lib()
    dev = torch.device("cuda", 0)
    mol = water_cluster(3, seed=21)
    other = water_cluster(3, seed=22)             # same shells, other geometry: valid data either way
    inp = _Inputs(mol, pinned=True)
    n = mol.n_bf
    out = [torch.full((n, n), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
    s = torch.cuda.Stream(dev)
    # queue slow work first so that the call's copies would still be pending if they read the caller's arrays
    big = torch.empty(1 << 26, dtype=torch.float64, device=dev)
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(s):
        for _ in range(20):
            big.mul_(1.0000001)
    rc = _call(L, inp, out, s)
    assert rc == 0, L.tf_error_string(rc)
    inp.xyz[...] = np.asarray(other.xyz)          # overwrite right after the call returns
    inp.ex *= 1.25
    inp.co *= 0.5
    s.synchronize()
    _check(out, mol)


@pytest.mark.gpu
def test_noalloc_rejects_oversized_input(cuda_ok):
    import torch
    L = _lib()
    mol = water_cluster(24, seed=1)            # 576 functions > 512
    inp = _Inputs(mol)
    n = mol.n_bf
    # full-size outputs, so that even a missed size check could not write out of bounds
    out = [torch.zeros((n, n), dtype=torch.float64, device="cuda:0") for _ in range(3)]
    rc = _call(L, inp, out)
    torch.cuda.synchronize()
    assert rc == TF_EUNSUPPORTED
    assert all(float(t.abs().max()) == 0.0 for t in out)


@pytest.mark.gpu
def test_noalloc_rejects_too_many_primitives(cuda_ok):
    """4200 primitives in 20 s shells: within the 512 Cartesian functions, beyond the
    4096 primitives of the scratch array."""
    import torch
    from tonto_b200.fock import _Basis
    L = _lib()
    n_shell, nprim = 20, 210
    xyz = np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 1.4]])
    Z = np.array([1.0, 1.0])
    sa = np.array([s % 2 for s in range(n_shell)], dtype=np.int32)
    sl = np.zeros(n_shell, dtype=np.int32)
    sn = np.full(n_shell, nprim, dtype=np.int32)
    sf = np.arange(n_shell, dtype=np.int32)
    ex = np.geomspace(0.05, 500.0, n_shell * nprim)
    co = np.full(n_shell * nprim, 0.01)
    basis = _Basis(2, _dp(xyz), n_shell, _ip(sa), _ip(sl), _ip(sn), _ip(sf), _dp(ex), _dp(co), 1)
    out = [torch.zeros((n_shell, n_shell), dtype=torch.float64, device="cuda:0") for _ in range(3)]
    rc = L.tf_one_electron_noalloc(ctypes.byref(basis), _dp(Z), *[ctypes.c_void_p(t.data_ptr()) for t in out], None)
    torch.cuda.synchronize()
    assert rc == TF_EUNSUPPORTED
    assert all(float(t.abs().max()) == 0.0 for t in out)


@pytest.mark.gpu
def test_noalloc_rejects_host_output_arrays(cuda_ok):
    import torch
    L = _lib()
    mol = water_cluster(2, seed=3)
    inp = _Inputs(mol)
    n = mol.n_bf
    host = np.zeros((n, n))
    dev_out = [torch.zeros((n, n), dtype=torch.float64, device="cuda:0") for _ in range(2)]
    rc = L.tf_one_electron_noalloc(ctypes.byref(inp.basis), _dp(inp.Z), ctypes.c_void_p(host.ctypes.data),
                                   *[ctypes.c_void_p(t.data_ptr()) for t in dev_out], None)
    torch.cuda.synchronize()
    assert rc == TF_EINVAL
    assert float(np.abs(host).max()) == 0.0
