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
