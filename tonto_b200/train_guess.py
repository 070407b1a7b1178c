"""Train and evaluate the learned initial density for water clusters.

    python -m tonto_b200.train_guess [--n-train 2000] [--n-test 200] [--epochs 300]
                                     [--out tonto_b200/data/guess_mlp.npz]
    python -m tonto_b200.train_guess --eval-only --n-test 20

Training data: converged RHF densities (cc-pVDZ, spherical, |dE| < 1e-8) of seeded
clusters with n uniform in [2, 16] (cluster seeds 100000 + i), produced by this
package's own SCF on the GPU.  Held-out evaluation clusters: n uniform in [8, 32]
(seeds 500000 + i).  For each held-out cluster the SCF is run from the core guess,
the monomer-superposition guess and the learned guess (with fallback to the
superposition guess if the DIIS error has not fallen after 3 cycles); iterations
and wall time to |dE| < 1e-8 are reported.
"""

from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import guess as G
from . import learned_guess as LG
from .molecules import water_cluster

TRAIN_SEED0, TEST_SEED0 = 100000, 500000


def monomer_density(device: int = 0) -> np.ndarray:
    import torch
    from .scf import RHF
    ref = G.reference_water()
    r = RHF(ref, schwarz_cutoff=1e-12, device=device).run(conv=1e-11, diis_tol=1e-8)
    _, _, A = G.cluster_rotations(ref)
    return G.to_local(r.P.cpu().numpy(), A[0], A[0])


def cluster_sizes(n_clusters: int, lo: int, hi: int, seed: int) -> np.ndarray:
    return np.random.default_rng(seed).integers(lo, hi + 1, size=n_clusters)


def generate(n_train: int, P_mono: np.ndarray, device: int = 0, log=print, env_k: int = LG.ENV_K):
    import torch
    from .scf import RHF
    Xs, Ys = [], []
    sizes = cluster_sizes(n_train, 2, 16, 7)
    t0 = time.time()
    for i, n in enumerate(sizes):
        mol = water_cluster(int(n), seed=TRAIN_SEED0 + i)
        rhf = RHF(mol, schwarz_cutoff=1e-12, device=device)
        P0 = torch.tensor(G.superposition_guess(mol, P_mono), device=rhf.dev)
        r = rhf.run(P0=P0, conv=1e-8, diis_tol=1e-5)
        ws, frames, A, atoms = LG.cluster_geometry(mol)
        pairs = LG.pair_list(atoms)
        Xs.append(LG.descriptors(atoms, frames, pairs, env_k))
        Ys.append(LG.local_blocks(mol, r.P.cpu().numpy(), A, pairs, P_mono))
        rhf.fb.close()
        if (i + 1) % 100 == 0:
            log(f"  generated {i + 1}/{n_train} clusters ({time.time() - t0:.0f} s)")
    return np.concatenate(Xs), np.concatenate(Ys)


def train(X: np.ndarray, Y: np.ndarray, epochs: int, device: int = 0, batch: int = 512, lr: float = 2e-3,
          seed: int = 0, log=print) -> LG.MLP:
    import torch
    model = LG.MLP(X.shape[1], Y.shape[1], device=device, seed=seed)
    model.x_mean = X.mean(0)
    model.x_std = np.maximum(X.std(0), 1e-3)
    # one global output scale: the loss then weighs every density element by its
    # absolute error, which is what the SCF starting point cares about
    model.y_mean = Y.mean(0)
    model.y_std = np.full(Y.shape[1], max(float((Y - model.y_mean).std()), 1e-6))
    Xn = torch.tensor((X - model.x_mean) / model.x_std, dtype=torch.float32, device=model.dev)
    Yn = torch.tensor((Y - model.y_mean) / model.y_std, dtype=torch.float32, device=model.dev)
    n = Xn.shape[0]
    rng = np.random.default_rng(seed)
    steps_per_epoch = max(1, n // batch)
    total = epochs * steps_per_epoch
    step = 0
    for ep in range(epochs):
        perm = torch.tensor(rng.permutation(n), device=model.dev)
        tot = 0.0
        for b in range(steps_per_epoch):
            idx = perm[b * batch:(b + 1) * batch]
            xb, yb = Xn[idx].contiguous(), Yn[idx].contiguous()
            out = model.forward(xb, keep=True)
            loss, dY = model.mse(out, yb)
            model.backward(dY)
            cur = lr * 0.5 * (1.0 + np.cos(np.pi * step / total))
            model.adam(cur, weight_decay=1e-6)
            tot += float(loss) if b == steps_per_epoch - 1 else 0.0
            step += 1
        if ep % max(1, epochs // 10) == 0 or ep == epochs - 1:
            log(f"  epoch {ep:4d} loss {tot:.4e}")
    return model


# The SCF schedule of the fast evaluation: mixed-precision quartets below the Schwarz x
# density bound 1e-6, incremental builds with a cutoff of 1e-4 x the DIIS error (at most
# 1e-10), and full FP64 builds at the tight cutoff in the final cycles.
FAST_SCF = {"mixed": True, "incremental": True, "loosen": 1e-4, "loose_max": 1e-10}


def evaluate(model: LG.MLP, P_mono: np.ndarray, n_test: int, device: int = 0, conv: float = 1e-8, log=print,
             fast: bool = False):
    import torch
    from .scf import RHF
    sizes = cluster_sizes(n_test, 8, 32, 11)
    rows = []
    for i, n in enumerate(sizes):
        mol = water_cluster(int(n), seed=TEST_SEED0 + i)
        rhf = RHF(mol, schwarz_cutoff=1e-12, device=device)
        res = {"n": int(n)}
        P_sup = torch.tensor(G.superposition_guess(mol, P_mono), device=rhf.dev)
        t = time.perf_counter()
        P_learn = torch.tensor(LG.learned_density(mol, model, P_mono), device=rhf.dev)
        t_pred = time.perf_counter() - t
        for name, P0, fb in (("core", None, None), ("superposition", P_sup, None),
                             ("learned", P_learn, lambda: P_sup)):
            r = rhf.run(P0=P0, conv=conv, diis_tol=1e-5, fallback=fb, **(FAST_SCF if fast else {}))
            res[name] = {"iterations": r.iterations, "seconds": r.seconds + (t_pred if name == "learned" else 0.0),
                         "energy": r.energy, "converged": r.converged, "fell_back": r.fell_back,
                         "first_diis_error": r.history[0][3]}
        res["learned"]["energy_diff_vs_core"] = res["learned"]["energy"] - res["core"]["energy"]
        rows.append(res)
        rhf.fb.close()
        log(f"  test {i}: n={n} it core/sup/learned = {res['core']['iterations']}/"
            f"{res['superposition']['iterations']}/{res['learned']['iterations']}")
    summ = {}
    for name in ("core", "superposition", "learned"):
        summ[name] = {"mean_iterations": float(np.mean([r[name]["iterations"] for r in rows])),
                      "mean_seconds": float(np.mean([r[name]["seconds"] for r in rows])),
                      "mean_first_diis_error": float(np.mean([r[name]["first_diis_error"] for r in rows])),
                      "all_converged": all(r[name]["converged"] for r in rows)}
    summ["learned"]["fallbacks"] = int(sum(r["learned"]["fell_back"] for r in rows))
    summ["learned"]["max_abs_energy_diff_vs_core"] = float(max(abs(r["learned"]["energy_diff_vs_core"])
                                                               for r in rows))
    return summ, rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-train", type=int, default=2000)
    ap.add_argument("--n-test", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--out", default=LG.DEFAULT_WEIGHTS)
    ap.add_argument("--data", default=None, help="cache of the generated training set (.npz)")
    ap.add_argument("--report", default=None, help="write the evaluation summary (JSON)")
    ap.add_argument("--eval-only", action="store_true")
    ap.add_argument("--env-k", type=int, default=LG.ENV_K, help="environment waters in the pair descriptor")
    ap.add_argument("--fast", action="store_true",
                    help="evaluate with mixed-precision incremental builds (FAST_SCF) instead of plain FP64 builds")
    args = ap.parse_args()
    P_mono = monomer_density()
    if args.eval_only:
        model = LG.MLP.load(args.out)
    else:
        t0 = time.time()
        if args.data and os.path.exists(args.data):
            z = np.load(args.data)
            X, Y = z["X"], z["Y"]
        else:
            X, Y = generate(args.n_train, P_mono, env_k=args.env_k)
            if args.data:
                np.savez_compressed(args.data, X=X, Y=Y)
        print(f"training set: {X.shape[0]} pair blocks from {args.n_train} clusters ({time.time() - t0:.0f} s)")
        t0 = time.time()
        model = train(X, Y, args.epochs)
        print(f"trained in {time.time() - t0:.0f} s")
        os.makedirs(os.path.dirname(args.out), exist_ok=True)
        model.save(args.out, extra={"mono_P_local": P_mono, "meta_n_train": np.array(args.n_train),
                                    "meta_epochs": np.array(args.epochs)})
    summ, rows = evaluate(model, P_mono, args.n_test, fast=args.fast)
    print(json.dumps(summ, indent=1))
    if args.report:
        with open(args.report, "w") as fh:
            json.dump({"summary": summ, "clusters": rows}, fh, indent=1)


if __name__ == "__main__":
    main()
