"""Frequency sharding across ranks: every point swept exactly once and the gather
restores sweep order (CPU, gloo, world size 2)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from sawsim_b200.shard import gather_charges, shard


def test_shards_partition_the_sweep():
    for n in (1, 7, 201, 402):
        for world in (1, 2, 3, 8):
            idx = np.concatenate([shard(n, r, world) for r in range(world)])
            assert np.array_equal(np.sort(idx), np.arange(n))


def _free_port():
    s = socket.socket()
    s.bind(('127.0.0.1', 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, n, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        f = np.linspace(1.6e9, 2.0e9, n)
        idx = shard(n, rank, world)
        Q = (f[idx] * 1e-9) + 1j * idx          # stand-in for the sweep's charges
        full = gather_charges(Q, n, rank, world)
        out[rank] = bool(np.array_equal(full, f * 1e-9 + 1j * np.arange(n)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize('n', [201, 8])
def test_gather_restores_order_gloo(n):
    ctx = mp.get_context('spawn')
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(2, _free_port(), n, out), nprocs=2, start_method='spawn')
        assert out[0] and out[1]
