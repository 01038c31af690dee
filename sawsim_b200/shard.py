"""Frequency sharding across GPUs (one process per GPU).

Every frequency point is independent once the pattern and the symbolic analysis
exist, so a sweep shards by points with no collective on the data path: rank r
of N takes the points r, r + N, r + 2N, ... of the sweep (interleaved, so that
every rank sees the whole band and the same mix of easy and near-resonant
points), builds its own engine (assembly and analysis are replicated: they are
cheap next to the factorisations), and the charges are gathered once at the
end.  This replaces the reference's fork pool over frequencies
(src/sawsim/frequency_tasks.py:33-55), which shares nothing but the assembled
matrices either.
"""
from __future__ import annotations

import numpy as np


def shard(n_points: int, rank: int, world: int) -> np.ndarray:
    """Indices of the points that ``rank`` of ``world`` sweeps."""
    if not 0 <= rank < world:
        raise ValueError('rank out of range')
    return np.arange(rank, n_points, world)


def gather_charges(Q_local: np.ndarray, n_points: int, rank: int, world: int):
    """All-gather the complex charges of every rank into sweep order (all ranks
    receive the full vector).  Uses the default torch.distributed group; one
    collective per sweep."""
    import torch
    import torch.distributed as dist
    if world == 1:
        return np.asarray(Q_local)
    width = (n_points + world - 1) // world
    buf = np.zeros((width, 2))
    buf[:len(Q_local), 0] = np.real(Q_local)
    buf[:len(Q_local), 1] = np.imag(Q_local)
    dev = 'cuda' if dist.get_backend() == 'nccl' else 'cpu'
    t = torch.from_numpy(buf).to(dev)
    parts = [torch.zeros_like(t) for _ in range(world)]
    dist.all_gather(parts, t)
    out = np.zeros(n_points, dtype=complex)
    for r, p in enumerate(parts):
        idx = shard(n_points, r, world)
        a = p.cpu().numpy()[:idx.size]
        out[idx] = a[:, 0] + 1j * a[:, 1]
    return out
