"""Column sharding across ranks (gloo, world size 2, CPU): each rank transforms its block
of columns (with the oracle, on the CPU) and the all-gathered result equals the unsharded
transform."""
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
