"""Failure handling on the GPU, made on the host without faulting the device:

* a density with a NaN or infinite element is refused with TF_EINVAL (the maxima
  kernel flags it and the list passes list nothing), on the host and device entry
  points, graph and class-by-class builds; the context stays usable;
* every device allocation of context creation and of the first builds is made to
  fail in turn (tf_debug_fail_alloc, a fake out-of-memory), and each must come back
  as TF_ENOMEM, never as a wrong J or K; afterwards the context builds correctly.
"""

import ctypes
import math

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster

TF_EINVAL, TF_ENOMEM = -1, -3
TOL = 1e-11


def _core_density(orc, mol, oracle_mod):
    S, T, V = orc.one_electron()
    P, _, _ = oracle_mod.density_from_fock(T + V, oracle_mod.orthogonaliser(S), mol.n_electrons // 2)
    return P


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [math.nan, math.inf, -math.inf])
def test_nonfinite_density_is_refused(cuda_ok, oracle_mod, bad):
    import torch
    from tonto_b200.fock import FockBuilder, TontoFockError
    mol = water_cluster(2, seed=0)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P = _core_density(orc, mol, oracle_mod)
    Jr, Kr = orc.jk(P)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    Pbad = P.copy()
    Pbad[3, 7] = Pbad[7, 3] = bad
    for graph in (False, True):
        fb.set_graph(graph)
        fb.make_r_JK(P)                                   # a good build first (sizes the graph buffers)
        with pytest.raises(TontoFockError, match="-1"):
            fb.make_r_JK(Pbad)
        # the device entry point refuses it too
        dev = torch.device("cuda", 0)
        Pd = torch.tensor(np.ascontiguousarray(Pbad.T), device=dev)
        Jd = torch.empty_like(Pd)
        Kd = torch.empty_like(Pd)
        with pytest.raises(TontoFockError, match="-1"):
            fb.make_r_JK_device(Pd, Jd, Kd)
        J, K = fb.make_r_JK(P)                            # and the context is still usable
        assert np.max(np.abs(J - Jr)) <= TOL and np.max(np.abs(K - Kr)) <= TOL


@pytest.mark.gpu
def test_injected_allocation_failures_return_enomem(cuda_ok, oracle_mod):
    from tonto_b200.fock import _Basis, _basis_struct, load_library, default_options
    L = load_library()
    mol = water_cluster(2, seed=1)
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    P = np.asfortranarray(_core_density(orc, mol, oracle_mod))
    Jr, Kr = orc.jk(P)
    keep = []
    basis = _basis_struct(mol, keep)
    opt = default_options(eri_schwarz_cutoff=1e-12)
    n = mol.n_bf
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    failures = 0
    try:
        for k in range(1, 200):
            L.tf_debug_fail_alloc(k)
            h = ctypes.c_void_p()
            rc = L.tf_ctx_create(ctypes.byref(basis), ctypes.byref(opt), ctypes.byref(h))
            built = True
            if rc == 0:
                J = np.full((n, n), np.nan, order="F")
                K = np.full((n, n), np.nan, order="F")
                for _ in range(3):                        # first builds: list, scan scratch, graph
                    rb = L.tf_build_jk(h, dp(P), dp(J), dp(K), 0)
                    assert rb in (0, TF_ENOMEM), rb
                    if rb == TF_ENOMEM:
                        failures += 1
                        built = False
                        break
                    # a build that reports success is right
                    assert np.max(np.abs(J - Jr)) <= TOL and np.max(np.abs(K - Kr)) <= TOL
                L.tf_debug_fail_alloc(0)
                if not built:                             # the context recovers once memory is there
                    rb = L.tf_build_jk(h, dp(P), dp(J), dp(K), 0)
                    assert rb == 0
                    assert np.max(np.abs(J - Jr)) <= TOL and np.max(np.abs(K - Kr)) <= TOL
                L.tf_ctx_destroy(h)
                if built:
                    break                                 # the countdown outran every allocation
            else:
                assert rc == TF_ENOMEM, rc
                assert not h.value
                failures += 1
        assert failures >= 10                            # creation and first builds allocate many buffers
    finally:
        L.tf_debug_fail_alloc(0)
