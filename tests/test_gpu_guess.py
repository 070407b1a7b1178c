"""Learned-guess network: CUDA gradients against the float64 CPU oracle, and the
guess's effect on SCF iterations."""

import os

import numpy as np
import pytest


@pytest.mark.gpu
def test_mlp_gradients_match_cpu_oracle(cuda_ok):
    import torch
    import mlp_oracle
    from tonto_b200.learned_guess import MLP
    rng = np.random.default_rng(0)
    B, d_in, d_out, width = 37, 51, 70, 40
    m = MLP(d_in, d_out, width=width, seed=3)
    for p in m.params[1::2]:                      # nonzero biases
        p.copy_(torch.tensor(rng.normal(size=p.shape) * 0.1, dtype=torch.float32))
    X = rng.normal(size=(B, d_in))
    T = rng.normal(size=(B, d_out))
    w = rng.uniform(0.5, 2.0, size=B)
    Xt = torch.tensor(X, dtype=torch.float32, device="cuda")
    Tt = torch.tensor(T, dtype=torch.float32, device="cuda")
    wt = torch.tensor(w, dtype=torch.float32, device="cuda")
    Y = m.forward(Xt, keep=True)
    loss, dY = m.mse(Y, Tt, wt)
    grads = m.backward(dY)
    params64 = [p.double().cpu().numpy() for p in m.params]
    Yr, _ = mlp_oracle.forward(params64, X)
    lr, gr = mlp_oracle.loss_and_grads(params64, X, T, w)
    assert np.max(np.abs(Y.cpu().numpy() - Yr)) < 1e-4 * max(1.0, np.abs(Yr).max())
    assert abs(float(loss) - lr) < 1e-5 * lr
    for g, r in zip(grads, gr):
        g = g.cpu().numpy()
        assert np.max(np.abs(g - r)) <= 2e-4 * np.max(np.abs(r)) + 1e-7


@pytest.mark.gpu
def test_adam_reduces_loss(cuda_ok):
    import torch
    from tonto_b200.learned_guess import MLP
    rng = np.random.default_rng(1)
    X = torch.tensor(rng.normal(size=(256, 8)), dtype=torch.float32, device="cuda")
    T = torch.tensor(np.sin(rng.normal(size=(256, 3))), dtype=torch.float32, device="cuda")
    m = MLP(8, 3, width=32, seed=0)
    first = None
    for _ in range(300):
        Y = m.forward(X, keep=True)
        loss, dY = m.mse(Y, T)
        m.backward(dY)
        m.adam(3e-3)
        first = float(loss) if first is None else first
    assert float(loss) < 0.2 * first


@pytest.mark.gpu
def test_trained_guess_cuts_scf_cycles_not_the_answer(cuda_ok):
    """The committed network (tonto_b200/data/guess_mlp.npz) on held-out clusters (seeds
    outside the training range), against the core guess and against the superposition of
    isolated-water densities it falls back to: a density closer to the converged one
    than the superposition's (smaller largest element error, smaller DIIS error of the
    first cycle), no more SCF cycles than from the superposition, far fewer than from
    the core guess, and the same converged energy."""
    import torch
    from tonto_b200 import guess as G
    from tonto_b200 import learned_guess as LG
    from tonto_b200.molecules import water_cluster
    from tonto_b200.scf import RHF
    model = LG.MLP.load()
    P_mono = model.extra["mono_P_local"]
    for i, n in enumerate((8, 11)):
        mol = water_cluster(n, seed=900000 + i)
        rhf = RHF(mol, schwarz_cutoff=1e-12)
        core = rhf.run(conv=1e-8, diis_tol=1e-5)
        P_sup = torch.tensor(G.superposition_guess(mol, P_mono), device=rhf.dev)
        P0 = torch.tensor(LG.learned_density(mol, model, P_mono), device=rhf.dev)
        learned = rhf.run(P0=P0, conv=1e-8, diis_tol=1e-5, fallback=lambda: P_sup)
        sup = rhf.run(P0=P_sup, conv=1e-8, diis_tol=1e-5)
        assert core.converged and learned.converged and sup.converged and not learned.fell_back
        assert learned.iterations <= 0.7 * core.iterations, (learned.iterations, core.iterations)
        assert learned.iterations <= sup.iterations, (learned.iterations, sup.iterations)
        err_l, err_s = float((P0 - core.P).abs().max()), float((P_sup - core.P).abs().max())
        assert err_l < 0.8 * err_s, (err_l, err_s)
        assert learned.history[0][3] < 0.8 * sup.history[0][3], (learned.history[0][3], sup.history[0][3])
        assert abs(learned.energy - core.energy) < 1e-8 and abs(sup.energy - core.energy) < 1e-8
