"""World-size-2 gloo test of the column-sharded multi-rank solve (CPU: the per-rank
solver is the oracle, standing in for the device solve each GPU rank runs)."""

import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from amjax_b200.distributed import shard_columns, solve_sharded


def test_shard_columns_partition():
    for k in (1, 5, 64, 65):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                lo, hi = shard_columns(k, world, r)
                seen += list(range(lo, hi))
            assert seen == list(range(k))
    with pytest.raises(ValueError):
        shard_columns(4, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from oracle import amg_oracle as O
    from tests.helpers import host_hierarchy, oracle_ml
    host = host_hierarchy("sa", 16)
    oml = oracle_ml(host)
    B = torch.as_tensor(np.random.default_rng(0).standard_normal((256, 5)))

    def solve_fn(Bl, tol, maxiter):
        cols = [O.solve(oml, Bl[:, c].numpy(), tol=tol, maxiter=maxiter)[0] for c in range(Bl.shape[1])]
        return torch.as_tensor(np.stack(cols, axis=1))

    X = solve_sharded(None, B, solve_fn=solve_fn, tol=1e-10, maxiter=100)
    if rank == 0:
        np.save(os.path.join(out_dir, "X.npy"), X.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_solve(tmp_path):
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    X = np.load(tmp_path / "X.npy")
    from oracle import amg_oracle as O
    from tests.helpers import host_hierarchy, oracle_ml
    host = host_hierarchy("sa", 16)
    oml = oracle_ml(host)
    B = np.random.default_rng(0).standard_normal((256, 5))
    for c in range(5):
        xo = O.solve(oml, B[:, c], tol=1e-10, maxiter=100)[0]
        np.testing.assert_allclose(X[:, c], xo, rtol=1e-12, atol=1e-14)
