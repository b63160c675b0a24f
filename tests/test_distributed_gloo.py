"""Multi-rank plumbing of the sharded signature batch, on CPU with gloo
(world size 2): shards tile the batch and balance total length, and the
all-gathered result equals the single-process one.  The per-rank compute is
the CPU oracle here (the GPU kernel is covered by the -m gpu tests)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from roughpy_b200.distributed import shard_bounds


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_shard_bounds_tile_and_balance():
    rng = np.random.default_rng(2)
    lens = rng.integers(16, 4097, size=4096)
    off = np.zeros(lens.size + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    for world in (1, 2, 3, 8):
        b = shard_bounds(off, world)
        assert b[0][0] == 0 and b[-1][1] == lens.size
        for (l0, h0), (l1, h1) in zip(b, b[1:]):
            assert h0 == l1
        loads = [int(off[h] - off[l]) for l, h in b]
        assert max(loads) - min(loads) <= 2 * int(lens.max())
    # one stream over four ranks: exactly one rank owns it
    one = shard_bounds(np.array([0, 5]), 4)
    assert sum(h - l for l, h in one) == 1 and one[-1][1] == 1


def _worker(rank, world, port, result_path):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import oracle
        from roughpy_b200.distributed import sharded_signatures
        rng = np.random.default_rng(0)
        lens = rng.integers(0, 20, size=13)
        off = np.zeros(lens.size + 1, dtype=np.int64)
        np.cumsum(lens, out=off[1:])
        inc = rng.normal(0, 0.3, size=(int(off[-1]), 3))

        def compute(rows, local_off):
            return torch.from_numpy(oracle.signatures(3, 3, rows, local_off))

        full = sharded_signatures(inc, off, 3, 3, "f64", compute=compute)
        if rank == 0:
            np.save(result_path, full.numpy())
    finally:
        dist.destroy_process_group()


def test_sharded_signatures_gloo_world_2(tmp_path):
    import oracle
    port = _free_port()
    out = str(tmp_path / "full.npy")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    rng = np.random.default_rng(0)
    lens = rng.integers(0, 20, size=13)
    off = np.zeros(lens.size + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    inc = rng.normal(0, 0.3, size=(int(off[-1]), 3))
    np.testing.assert_allclose(got, oracle.signatures(3, 3, inc, off), rtol=0, atol=1e-14)
