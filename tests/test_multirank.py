"""Multi-rank sharding of the K build (CPU, gloo, world size 2).

Set quartets are independent and K is additive, so each rank builds K over its strided share
and one all-reduce sums the partial K. Here the ranks run the oracle; the engine follows the
same split in bench.py.
"""
import os
import socket

import numpy as np
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


def test_two_rank_sharded_K_equals_single(tmp_path):
    out = str(tmp_path / "k.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn", join=True)
    from libgint_b200.workload import Api, Session, Workload
    w = Workload("small_l2")
    K1 = Session(Api(ORACLE_SO), w).build_K()[0]
    K2 = np.load(out)
    assert np.abs(K1 - K2).max() <= 1e-12 * np.abs(K1).max()
