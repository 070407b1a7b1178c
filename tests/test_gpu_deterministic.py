"""Deterministic builds (tf_options.deterministic = 1).  Every J/K contribution is
added as two 64-bit fixed-point words with integer atomics, whose sums do not
depend on the order of the additions, so one density gives the same bits on every
path a build can take: class by class or as a replayed graph, any kernel variant,
any graph-branch schedule the autotuner picks, a chunked quartet list, the list
written with or without the screening record.  Tonto's serial loop
(molecule.fock.foo:1274-1361) is bitwise reproducible for a fixed rank count; these
builds are too, and still match the oracle to the FP64 bar."""

import numpy as np
import pytest

from tonto_b200.molecules import water_cluster

TOL = 1e-11


def _density(mol, seed, scale=0.03):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(mol.n_bf, mol.n_bf)) * scale
    return A + A.T


def _same(a, b):
    return all(np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.gpu
def test_bits_do_not_depend_on_the_build_path(cuda_ok, oracle_mod):
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(6, seed=11)
    P = _density(mol, 5)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12, deterministic=True)
    fb.set_graph(False)
    ref = fb.make_r_JK(P)
    runs = {"again": fb.make_r_JK(P)}
    for v in range(4):
        fb.set_kernel_variant(v)
        runs["variant %d" % v] = fb.make_r_JK(P)
    fb.set_list_budget(1 << 16)                    # the list in many chunks
    runs["chunked"] = fb.make_r_JK(P)
    fb.set_screen_record_budget(0)                 # the list write screens again
    runs["no record"] = fb.make_r_JK(P)
    fb.set_list_budget(1 << 30)
    fb.set_screen_record_budget(1 << 33)
    fb.set_graph(True)
    runs["graph capture"] = fb.make_r_JK(P)
    runs["graph replay"] = fb.make_r_JK(P)
    fb.close()
    for name, r in runs.items():
        assert _same(r, ref), name
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    Jr, Kr = orc.jk(P)
    assert np.max(np.abs(ref[0] - Jr)) <= TOL
    assert np.max(np.abs(ref[1] - Kr)) <= TOL
    plain = FockBuilder(mol, schwarz_cutoff=1e-12)
    J, K = plain.make_r_JK(P)
    plain.close()
    assert np.max(np.abs(ref[0] - J)) <= 1e-12 and np.max(np.abs(ref[1] - K)) <= 1e-12


@pytest.mark.gpu
def test_bits_do_not_depend_on_the_autotuned_schedule(cuda_ok):
    import torch
    from tonto_b200.fock import TF_JK_MIXED, FockBuilder
    mol = water_cluster(8, seed=12)
    P = torch.tensor(_density(mol, 6), device="cuda:0").contiguous()
    J = torch.empty_like(P)
    K = torch.empty_like(P)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12, deterministic=True)
    for flags in (0, TF_JK_MIXED):
        fb.make_r_JK_device(P, J, K, flags)
        torch.cuda.synchronize()
        ref = (J.clone(), K.clone())
        fb.autotune(P, J, K, flags, max_streams=4)   # variants and graph branches by timing
        for _ in range(2):
            fb.make_r_JK_device(P, J, K, flags)
            torch.cuda.synchronize()
            assert torch.equal(J, ref[0]) and torch.equal(K, ref[1])
    fb.close()


@pytest.mark.gpu
def test_unrestricted_and_f_shell_builds(cuda_ok, oracle_mod):
    """The beta accumulators, and the warp kernel of the f-shell classes (cc-pVTZ)."""
    from tonto_b200.fock import FockBuilder
    mol = water_cluster(1, seed=6, basis="cc-pVTZ")
    Pa, Pb = _density(mol, 3), _density(mol, 4)
    fb = FockBuilder(mol, schwarz_cutoff=1e-12, deterministic=True)
    fb.set_graph(False)
    a = fb.make_u_JK(Pa, Pb)
    fb.set_kernel_variant(3)
    b = fb.make_u_JK(Pa, Pb)
    assert _same(a, b)
    r = fb.make_r_JK(Pa)
    fb.close()
    orc = oracle_mod.Oracle(mol, schwarz_cutoff=1e-12)
    for x, y in zip(a, orc.jk_uhf(Pa, Pb)):
        assert np.max(np.abs(x - y)) <= TOL
    for x, y in zip(r, orc.jk(Pa)):
        assert np.max(np.abs(x - y)) <= TOL


@pytest.mark.gpu
def test_batched_context(cuda_ok, oracle_mod):
    from tonto_b200.fock import BatchFockBuilder
    mols = [water_cluster(n, seed=20 + n) for n in (1, 2, 3)]
    Ps = [_density(m, 30 + i) for i, m in enumerate(mols)]
    fb = BatchFockBuilder(mols, schwarz_cutoff=1e-12, deterministic=True)
    fb.set_graph(False)
    a = fb.make_r_JK_batched(Ps)
    fb.set_graph(True)
    b = fb.make_r_JK_batched(Ps)
    c = fb.make_r_JK_batched(Ps)
    fb.close()
    for i, m in enumerate(mols):
        assert _same((a[0][i], a[1][i]), (b[0][i], b[1][i])) and _same((a[0][i], a[1][i]), (c[0][i], c[1][i]))
        Jr, Kr = oracle_mod.Oracle(m, schwarz_cutoff=1e-12).jk(Ps[i])
        assert np.max(np.abs(a[0][i] - Jr)) <= TOL and np.max(np.abs(a[1][i] - Kr)) <= TOL
