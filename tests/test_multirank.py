"""Multi-rank sharding of the K build (gloo, world size 2).

Set quartets are independent and K is additive, so each rank builds K over its strided share
(set quartets rank, rank + world, ...: the split bench.py uses) and one all-reduce sums the partial
K. The CPU test runs the oracle on the ranks; the GPU test runs the engine in two processes on one
GPU (independent launches, nothing waits across processes) and sums their K with gloo.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ORACLE_SO, ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    from libgint_b200.workload import Api, Session, Workload
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = Workload("small_l2")
    nq = w.info["n_setq"]
    K, _, _ = Session(Api(ORACLE_SO), w).build_K_subset(np.arange(rank, nq, world))
    t = torch.from_numpy(K)
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


def _engine_worker(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import torch as _torch
    from libgint_b200.capi import engine_path
    from libgint_b200.workload import Api, Session, Workload
    _torch.cuda.set_device(0)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    w = Workload("periodic_l2", n_mol=3, box_ang=7.0, n_occ=20)
    nq = w.info["n_setq"]
    s = Session(Api(engine_path()), w)
    K, _, _ = s.build_K_subset(np.arange(rank, nq, world))
    s.close()
    t = torch.from_numpy(K)
    dist.all_reduce(t)
    if rank == 0:
        np.save(out, t.numpy())
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.gpu
def test_two_rank_engine_shards_sum_to_the_oracle_K(tmp_path):
    """The engine's data path under the bench's multi-GPU split: two ranks (processes) each build
    K over their strided share of the set quartets, a gloo all-reduce sums them, and the sum is the
    oracle's K of the whole list."""
    out = str(tmp_path / "ke.npy")
    mp.start_processes(_engine_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    from libgint_b200.workload import Api, Session, Workload
    w = Workload("periodic_l2", n_mol=3, box_ang=7.0, n_occ=20)
    Ko = Session(Api(ORACLE_SO), w).build_K()[0]
    Ke = np.load(out)
    rel = np.abs(Ke - Ko).max() / np.abs(Ko).max()
    print(f"2 engine ranks, summed K vs oracle: {rel:.3e}")
    assert rel <= 1e-12, rel


def test_two_rank_sharded_K_equals_single(tmp_path):
    out = str(tmp_path / "k.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    from libgint_b200.workload import Api, Session, Workload
    w = Workload("small_l2")
    K1 = Session(Api(ORACLE_SO), w).build_K()[0]
    K2 = np.load(out)
    assert np.abs(K1 - K2).max() <= 1e-12 * np.abs(K1).max()
