"""The no-allocation one-electron entry point, checked against the allocating one.

tf_one_electron_noalloc serves callers that cannot call cudaMalloc where they need
the integrals (a host framework that owns the GPU memory, or code where an
allocation is forbidden or would stall the device).  It keeps all scratch in one
fixed array in device memory and writes into arrays the caller already owns.  Two
calls in a row, on different molecules, must each match tf_one_electron.  This file
is collected last so that a failure here cannot stop the rest of the suite.
"""

import ctypes

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster

TOL = 1e-12


@pytest.mark.gpu
def test_noalloc_one_electron_matches_allocating_entry_point(cuda_ok):
    import torch
    from tonto_b200.fock import FockBuilder, _Basis, load_library

    L = load_library()
    L.tf_one_electron_noalloc.argtypes = [ctypes.POINTER(_Basis), ctypes.POINTER(ctypes.c_double),
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    dev = torch.device("cuda", 0)
    for mol in (water_cluster(2, seed=3), water_cluster(3, seed=5, spherical=False)):
        S0, T0, V0 = FockBuilder(mol).one_electron()
        n = mol.n_bf
        sa, sl, sn, sf, ex, co = mol.flat_arrays()
        xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64)
        Z = np.ascontiguousarray(mol.Z, dtype=np.float64)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))     # noqa: E731
        basis = _Basis(mol.n_atom, dp(xyz), mol.n_shell, ip(sa), ip(sl), ip(sn), ip(sf), dp(ex), dp(co),
                       int(mol.spherical))
        # caller-owned outputs, filled with garbage so that a missed element shows
        out = [torch.full((n, n), float("nan"), dtype=torch.float64, device=dev) for _ in range(3)]
        torch.cuda.synchronize(dev)
        rc = L.tf_one_electron_noalloc(ctypes.byref(basis), dp(Z), *[ctypes.c_void_p(t.data_ptr()) for t in out],
                                       None)
        assert rc == 0, L.tf_error_string(rc)
        torch.cuda.synchronize(dev)
        # outputs are column-major n x n; the matrices are symmetric
        for got, ref in zip(out, (S0, T0, V0)):
            g = got.cpu().numpy().T
            assert np.all(np.isfinite(g))
            assert np.max(np.abs(g - ref)) <= TOL


@pytest.mark.gpu
def test_noalloc_rejects_oversized_input(cuda_ok):
    import torch
    from tonto_b200.fock import _Basis, load_library
    L = load_library()
    L.tf_one_electron_noalloc.argtypes = [ctypes.POINTER(_Basis), ctypes.POINTER(ctypes.c_double),
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    mol = water_cluster(24, seed=1)            # 576 functions > 512
    sa, sl, sn, sf, ex, co = mol.flat_arrays()
    xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64)
    Z = np.ascontiguousarray(mol.Z, dtype=np.float64)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))     # noqa: E731
    basis = _Basis(mol.n_atom, dp(xyz), mol.n_shell, ip(sa), ip(sl), ip(sn), ip(sf), dp(ex), dp(co), 1)
    n = mol.n_bf
    # full-size outputs, so that even a missed size check could not write out of bounds
    out = [torch.zeros((n, n), dtype=torch.float64, device="cuda:0") for _ in range(3)]
    rc = L.tf_one_electron_noalloc(ctypes.byref(basis), dp(Z), *[ctypes.c_void_p(t.data_ptr()) for t in out], None)
    torch.cuda.synchronize()
    assert rc == -4    # TF_EUNSUPPORTED
    assert all(float(t.abs().max()) == 0.0 for t in out)
