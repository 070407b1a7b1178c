"""Sharded J/K builds on several ranks (gloo on CPU), with one all-reduce summing J
and K (PARALLEL_SYMMETRIC_SUM, molecule.fock.foo:1355-1357):

* the library's own shard plan (tf_plan_shards, the bra tasks tf_set_shard deals to
  each GPU by estimated cost; a host function, no GPU needed): every rank computes
  the plan, takes its tasks, expands them into their shell quartets and evaluates
  them with the oracle; the shares all-reduce to the full build, the plan is the
  same on every rank and its shards' estimated costs are even;
* Tonto's round-robin parallel do (FooToFortran.java:2762-2783): each rank takes
  every N-th bra shell pair of the oracle's loop.

On GPUs the same plan runs through tf_set_shard + an NCCL all-reduce in bench.py."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _plan(mol, max_I, cutoff, world):
    """The library's shard plan of one molecule (host call, no device)."""
    import ctypes
    from tonto_b200.fock import _Basis, _basis_struct, load_library
    L = load_library()
    keep = []
    basis = _basis_struct(mol, keep)
    mi = np.ascontiguousarray(max_I, dtype=np.float64)
    dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))     # noqa: E731
    nt = ctypes.c_longlong()
    rc = L.tf_plan_shards(ctypes.byref(basis), dp(mi), cutoff, world, ctypes.byref(nt), None, None, None, None, None,
                          None)
    assert rc == 0
    n = nt.value
    bra, kcls, klim, shard = (np.zeros(n, dtype=np.int32) for _ in range(4))
    pos = np.zeros(len(mi), dtype=np.int32)
    cost = np.zeros(world)
    rc = L.tf_plan_shards(ctypes.byref(basis), dp(mi), cutoff, world, ctypes.byref(nt), ip(bra), ip(kcls), ip(klim),
                          ip(shard), ip(pos), dp(cost))
    assert rc == 0
    return bra, kcls, klim, shard, pos, cost


def _pair_classes(mol):
    ls = [s.l for s in mol.shells]
    cls = []
    for a in range(len(ls)):
        for b in range(a + 1):
            h, lo = max(ls[a], ls[b]), min(ls[a], ls[b])
            cls.append(h * (h + 1) // 2 + lo)
    return np.array(cls)


def _expand(bra, kcls, klim, pos, pcls):
    """Shell quartets of a set of plan rows: the kets of the row's class at class-list
    positions up to the row's limit."""
    by_cls = {c: np.flatnonzero(pcls == c) for c in np.unique(pcls)}
    qb, qk = [], []
    for b, kc, lim in zip(bra, kcls, klim):
        kets = by_cls.get(int(kc), np.zeros(0, dtype=np.int64))
        kets = kets[pos[kets] <= lim]
        qb.append(np.full(len(kets), b))
        qk.append(kets)
    return np.concatenate(qb), np.concatenate(qk)


def _plan_worker(rank, world, port, q):
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle
    from tonto_b200.molecules import water_cluster
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mol = water_cluster(3, seed=17)
    cutoff = 1e-12
    orc = oracle.Oracle(mol, schwarz_cutoff=cutoff)
    S, T, V = orc.one_electron()
    P, _, _ = oracle.density_from_fock(T + V, oracle.orthogonaliser(S), mol.n_electrons // 2)
    bra, kcls, klim, shard, pos, cost = _plan(mol, orc.max_I(), cutoff, world)
    mine = shard == rank
    qb, qk = _expand(bra[mine], kcls[mine], klim[mine], pos, _pair_classes(mol))
    J, K = orc.jk_quartets(P, qb, qk, n_threads=1)
    Jt = torch.from_numpy(J.copy())
    Kt = torch.from_numpy(K.copy())
    dist.all_reduce(Jt)
    dist.all_reduce(Kt)
    plans = [torch.zeros(len(shard), dtype=torch.int32) for _ in range(world)]
    dist.all_gather(plans, torch.from_numpy(shard.copy()))
    nq = torch.tensor([len(qb)], dtype=torch.int64)
    dist.all_reduce(nq)
    if rank == 0:
        Jr, Kr = orc.jk(P, n_threads=1)
        # every unordered pair of shell pairs exactly once over the shards
        qa, qc = _expand(bra, kcls, klim, pos, _pair_classes(mol))
        key = np.maximum(qa, qc).astype(np.int64) * 10**6 + np.minimum(qa, qc)
        n_pairs = len(pos)
        q.put({"dJ": float(np.max(np.abs(Jt.numpy() - Jr))), "dK": float(np.max(np.abs(Kt.numpy() - Kr))),
               "same_plan": all(bool(torch.equal(p, plans[0])) for p in plans),
               "unique": len(np.unique(key)) == len(key) == n_pairs * (n_pairs + 1) // 2,
               "n_shard_quartets": int(nq.item()), "n_quartets": len(key),
               "imbalance": float(cost.max() / cost.mean() - 1.0)})
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_library_shard_plan_allreduces_to_full_build(oracle_mod, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_plan_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=60)
    assert res["dJ"] < 1e-12 and res["dK"] < 1e-12, res
    assert res["same_plan"] and res["unique"], res
    assert res["n_shard_quartets"] == res["n_quartets"], res
    assert res["imbalance"] < 0.02, res


def test_shard_plan_balances_estimated_cost():
    """On (H2O)8 at 4 shards the cost-balanced plan's largest shard is within 1 % of the
    mean estimated cost, and every shard gets tasks."""
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import oracle
    from tonto_b200.molecules import water_cluster
    mol = water_cluster(8, seed=2)
    orc = oracle.Oracle(mol, schwarz_cutoff=1e-12)
    bra, kcls, klim, shard, pos, cost = _plan(mol, orc.max_I(), 1e-12, 4)
    assert cost.max() / cost.mean() - 1.0 < 0.01
    assert sorted(np.unique(shard)) == [0, 1, 2, 3]


def _worker(rank, world, port, q):
    import sys
    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    import oracle
    from tonto_b200.molecules import water_cluster
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mol = water_cluster(2, seed=13)
    orc = oracle.Oracle(mol, schwarz_cutoff=1e-12)
    S, T, V = orc.one_electron()
    P, _, _ = oracle.density_from_fock(T + V, oracle.orthogonaliser(S), mol.n_electrons // 2)
    J, K = orc.jk_shard(P, rank, world, n_threads=1)
    Jt = torch.from_numpy(J.copy())
    Kt = torch.from_numpy(K.copy())
    dist.all_reduce(Jt)
    dist.all_reduce(Kt)
    if rank == 0:
        Jr, Kr = orc.jk(P, n_threads=1)
        q.put((float(np.max(np.abs(Jt.numpy() - Jr))), float(np.max(np.abs(Kt.numpy() - Kr)))))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_round_robin_shards_allreduce_to_full_build(oracle_mod, world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    dj, dk = q.get(timeout=240)
    for p in procs:
        p.join(timeout=60)
    assert dj < 1e-12 and dk < 1e-12
