"""Graph-captured builds: the same J and K as the class-by-class path, re-capture
when arrays or flags change, and the fall-back when a list outgrows the buffer."""

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster


@pytest.mark.gpu
def test_graph_builds_match_direct_builds(cuda_ok, oracle_mod):
    import torch
    from tonto_b200.fock import FockBuilder, TF_JK_MIXED
    mol = water_cluster(3, seed=5)
    n = mol.n_bf
    rng = np.random.default_rng(9)
    A = rng.normal(size=(n, n)) * 0.05
    P = A + A.T
    Jr, Kr = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk(P)

    direct = FockBuilder(mol, schwarz_cutoff=1e-12)
    direct.set_graph(False)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    dev = torch.device("cuda", 0)
    Pd = torch.tensor(np.ascontiguousarray(P.T), device=dev)
    J = torch.empty_like(Pd)
    K = torch.empty_like(Pd)
    seen = []
    for flags in (0, 0, 0, TF_JK_MIXED, TF_JK_MIXED, 0):
        fb.make_r_JK_device(Pd, J, K, flags)
        torch.cuda.synchronize()
        seen.append(fb.stats()["graph"])
        Jh, Kh = J.cpu().numpy().T, K.cpu().numpy().T
        tol = 1e-11 if flags == 0 else 1e-8
        assert np.max(np.abs(Jh - Jr)) < tol and np.max(np.abs(Kh - Kr)) < tol
    assert seen[0] == 0 and all(v == 1 for v in seen[1:])
    # host-buffer entry point, graph against class-by-class
    J1, K1 = fb.make_r_JK(P)
    J2, K2 = direct.make_r_JK(P)
    assert direct.stats()["graph"] == 0
    assert np.max(np.abs(J1 - J2)) < 1e-12 and np.max(np.abs(K1 - K2)) < 1e-12


@pytest.mark.gpu
def test_graph_list_overflow_falls_back(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(3, seed=6)
    n = mol.n_bf
    rng = np.random.default_rng(10)
    A = rng.normal(size=(n, n)) * 0.05
    P = A + A.T
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    # a tiny density sizes the list buffer small; the full density then overflows it
    fb.make_r_JK(P * 1e-9)
    fb.make_r_JK(P * 1e-9)
    assert fb.stats()["graph"] == 1
    J, K = fb.make_r_JK(P)
    assert fb.stats()["graph"] == 0
    Jr, Kr = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk(P)
    assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11
    J, K = fb.make_r_JK(P)
    assert fb.stats()["graph"] == 1
    assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11


@pytest.mark.gpu
def test_autotuned_schedule_keeps_results(cuda_ok, oracle_mod):
    import torch
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(4, seed=7)
    n = mol.n_bf
    rng = np.random.default_rng(11)
    A = rng.normal(size=(n, n)) * 0.05
    P = A + A.T
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    dev = torch.device("cuda", 0)
    Pd = torch.tensor(np.ascontiguousarray(P.T), device=dev)
    J = torch.empty_like(Pd)
    K = torch.empty_like(Pd)
    tune = fb.autotune(Pd, J, K, max_streams=3)
    assert 1 <= tune["streams"] <= 3 and tune["candidates"] == 3
    assert all(0.0 < t < 1e6 for t in tune["ms"])
    Jr, Kr = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk(P)
    for _ in range(2):
        fb.make_r_JK_device(Pd, J, K)
        torch.cuda.synchronize()
        assert fb.stats()["graph"] == 1
        assert np.max(np.abs(J.cpu().numpy().T - Jr)) < 1e-11 and np.max(np.abs(K.cpu().numpy().T - Kr)) < 1e-11


@pytest.mark.gpu
def test_every_kernel_variant_matches_oracle(cuda_ok, oracle_mod):
    """Each kernel variant the autotuner may choose (tf_set_kernel_variant 0 .. 3)
    gives the oracle's J and K; an out-of-range variant is refused."""
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(3, seed=8)
    n = mol.n_bf
    rng = np.random.default_rng(12)
    A = rng.normal(size=(n, n)) * 0.05
    P = A + A.T
    Jr, Kr = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk(P)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    for v in range(4):
        fb.set_kernel_variant(v)
        for _ in range(2):                       # first build direct, second from the graph
            J, K = fb.make_r_JK(P)
            assert np.max(np.abs(J - Jr)) < 1e-11 and np.max(np.abs(K - Kr)) < 1e-11, v
    from tonto_b200.fock import TontoFockError
    with pytest.raises(TontoFockError):
        fb.set_kernel_variant(4)


@pytest.mark.gpu
def test_rescreening_list_write_matches_record(cuda_ok, oracle_mod):
    """With no room for the screening record the list write screens again
    (tf_set_screen_record_budget 0); FP64 and mixed builds give the same J and K as
    with the record, and the same quartet counts, for one molecule and a batch."""
    from tonto_b200.fock import BatchFockBuilder, FockBuilder, TF_JK_MIXED
    mols = [water_cluster(3, seed=11), water_cluster(2, seed=12), water_cluster(4, seed=13)]
    rng = np.random.default_rng(14)
    Ps = []
    for m in mols:
        A = rng.normal(size=(m.n_bf, m.n_bf)) * 0.05
        Ps.append(A + A.T)
    Jr, Kr = oracle_mod.Oracle(mols[0], schwarz_cutoff=1e-12).jk(Ps[0])
    rec = FockBuilder(mols[0], schwarz_cutoff=1e-12, mixed_fp32_cut=1e-4)
    scr = FockBuilder(mols[0], schwarz_cutoff=1e-12, mixed_fp32_cut=1e-4)
    scr.set_screen_record_budget(0)
    for flags, tol in ((0, 1e-11), (TF_JK_MIXED, 1e-7)):
        for _ in range(2):                           # direct, then graph builds
            J1, K1 = rec.make_r_JK(Ps[0], flags)
            s1 = rec.stats()
            J2, K2 = scr.make_r_JK(Ps[0], flags)
            s2 = scr.stats()
            assert s1["quartets"] == s2["quartets"] and s1["quartets_fp32"] == s2["quartets_fp32"]
            assert np.max(np.abs(J2 - J1)) < 1e-12 and np.max(np.abs(K2 - K1)) < 1e-12
            assert np.max(np.abs(J2 - Jr)) < tol and np.max(np.abs(K2 - Kr)) < tol
    b1 = BatchFockBuilder(mols, schwarz_cutoff=1e-12, mixed_fp32_cut=1e-4)
    b2 = BatchFockBuilder(mols, schwarz_cutoff=1e-12, mixed_fp32_cut=1e-4)
    b2.set_screen_record_budget(0)
    for flags in (0, TF_JK_MIXED):
        Js1, Ks1 = b1.make_r_JK_batched(Ps, flags)
        Js2, Ks2 = b2.make_r_JK_batched(Ps, flags)
        assert b1.stats()["quartets"] == b2.stats()["quartets"]
        for a, b in zip(Js1 + Ks1, Js2 + Ks2):
            assert np.max(np.abs(a - b)) < 1e-12


@pytest.mark.gpu
def test_device_build_waits_for_the_callers_stream(cuda_ok, oracle_mod):
    """The density is written on torch's default (legacy, NULL) stream behind slow
    work, and the build is called at once: it must read the new density, not the
    buffer's old contents (the context's own stream does not synchronise with the
    legacy stream by itself)."""
    import torch
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(3, seed=15)
    n = mol.n_bf
    rng = np.random.default_rng(16)
    A = rng.normal(size=(n, n)) * 0.05
    P = A + A.T
    Jr, Kr = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12).jk(P)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12)
    dev = torch.device("cuda", 0)
    assert torch.cuda.current_stream(dev).cuda_stream == 0
    Pd = torch.zeros((n, n), dtype=torch.float64, device=dev)
    J = torch.empty_like(Pd)
    K = torch.empty_like(Pd)
    src = torch.tensor(np.ascontiguousarray(P.T), device=dev)
    big = torch.randn(4096, 4096, dtype=torch.float64, device=dev)
    for _ in range(2):                               # direct, then graph builds
        torch.cuda.synchronize()
        Pd.zero_()
        torch.cuda.synchronize()
        for _ in range(4):
            big = big @ big * 1e-3                   # tens of milliseconds ahead of the copy
        Pd.copy_(src)
        fb.make_r_JK_device(Pd, J, K)
        torch.cuda.synchronize()
        Jh, Kh = J.cpu().numpy().T, K.cpu().numpy().T
        assert np.max(np.abs(Jh - Jr)) < 1e-11 and np.max(np.abs(Kh - Kr)) < 1e-11
