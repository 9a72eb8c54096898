"""Sharding across ranks (gloo, world size 2, CPU), driving the library's sharding host logic
(nufht_b200.sharding) with the oracle standing in for each rank's GPU plan:

* column blocks: each rank transforms its block of columns and the all-gathered result equals
  the unsharded transform;
* target rows (fewer columns than ranks): each rank plans the sub-rectangle of its own target
  range against every source, receives c by broadcast, and the gathered rows equal the
  unsharded transform within the tolerance (the sub-plans partition their rectangles
  differently from the whole problem's plan)."""
import os
import socket

import numpy as np
import pytest

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out_path):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import oracle
    from nufht_b200.sharding import column_block, gather_columns
    rng = np.random.default_rng(0)
    r = np.sort(rng.uniform(0.01, 60, 1500))
    k = np.sort(rng.uniform(0.01, 40, 1200))
    c = rng.standard_normal((1500, 7))
    a, b = column_block(7, world, rank)
    g_local = oracle.nufht_batch(1.0, r, k, c[:, a:b], 1e-8)
    g = gather_columns(torch.from_numpy(np.ascontiguousarray(g_local)), 7)
    if rank == 0:
        np.save(out_path, g.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_column_blocks_cover_batch():
    from nufht_b200.sharding import column_block
    for total in (1, 7, 32, 33):
        for world in (1, 2, 3, 8):
            blocks = [column_block(total, world, r) for r in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == total
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
            assert max(b - a for a, b in blocks) - min(b - a for a, b in blocks) <= 1


def test_two_rank_gloo_column_sharding(tmp_path):
    import torch.multiprocessing as mp
    import oracle
    out = str(tmp_path / "g.npy")
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    g = np.load(out)
    rng = np.random.default_rng(0)
    r = np.sort(rng.uniform(0.01, 60, 1500))
    k = np.sort(rng.uniform(0.01, 40, 1200))
    c = rng.standard_normal((1500, 7))
    np.testing.assert_allclose(g, oracle.nufht_batch(1.0, r, k, c, 1e-8), rtol=0, atol=1e-12)


class _OraclePlan:
    """The oracle in place of DevicePlan (same execute_columns contract: (B, m) -> (B, n))."""

    def __init__(self, nu, r, k, tol):
        self.nu, self.r, self.k, self.tol = nu, np.asarray(r), np.asarray(k), tol

    def execute_columns(self, c_cols):
        import torch
        import oracle
        g = oracle.nufht_batch(self.nu, self.r, self.k, c_cols.numpy().T, self.tol)
        return torch.from_numpy(np.ascontiguousarray(g.T))


def _rows_worker(rank, world, port, out_path, nu, B):
    import sys
    sys.path.insert(0, ROOT)
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from nufht_b200.sharding import TargetShardedTransform, sharding_mode
    assert sharding_mode(B, world) == "targets"
    rng = np.random.default_rng(3)
    r = np.sort(rng.uniform(0.01, 80, 2500))
    k = np.sort(rng.uniform(0.01, 60, 2100))
    T = TargetShardedTransform(nu, r, k, 1e-8, make_plan=_OraclePlan)
    # only rank 0 holds the coefficients; the transform broadcasts them
    c = torch.from_numpy(rng.standard_normal((B, 2500))) if rank == 0 else torch.zeros((B, 2500), dtype=torch.float64)
    g = T(c, src=0)
    np.save(out_path + ".%d.npy" % rank, g.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_target_rows_cover_targets():
    from nufht_b200.sharding import target_rows, sharding_mode
    for n in (1, 5, 1000, 1001):
        for world in (1, 2, 4, 8):
            blocks = [target_rows(n, world, q) for q in range(world)]
            assert blocks[0][0] == 0 and blocks[-1][1] == n
            assert all(blocks[i][1] == blocks[i + 1][0] for i in range(world - 1))
    assert sharding_mode(32, 8) == "columns" and sharding_mode(1, 2) == "targets"


@pytest.mark.parametrize("nu,B", [(0.0, 1), (3.0, 1)])
def test_two_rank_gloo_target_row_sharding(tmp_path, nu, B):
    import torch.multiprocessing as mp
    import oracle
    out = str(tmp_path / "g")
    port = _free_port()
    mp.start_processes(_rows_worker, args=(2, port, out, nu, B), nprocs=2, join=True, start_method="spawn")
    rng = np.random.default_rng(3)
    r = np.sort(rng.uniform(0.01, 80, 2500))
    k = np.sort(rng.uniform(0.01, 60, 2100))
    c = rng.standard_normal((B, 2500))
    g_ref = oracle.nufht_batch(nu, r, k, c.T, 1e-8).T
    for q in range(2):
        g = np.load(out + ".%d.npy" % q)
        assert g.shape == (B, 2100)
        err = np.abs(g - g_ref).max(axis=1) / np.abs(c).sum(axis=1)
        assert err.max() <= 1e-8, (q, err)
