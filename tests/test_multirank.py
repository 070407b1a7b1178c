"""Sharded J/K build on several ranks (gloo on CPU): each rank takes every N-th bra
shell pair, as one MPI rank of Tonto's round-robin parallel do
(FooToFortran.java:2762-2783), and one all-reduce sums J and K
(PARALLEL_SYMMETRIC_SUM, molecule.fock.foo:1355-1357).  The same sharding runs on
GPUs through tf_set_shard + an NCCL all-reduce in bench.py."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


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
