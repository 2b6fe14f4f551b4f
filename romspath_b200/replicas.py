"""Particle sharding for runs on several GPUs (one process per GPU).

Particles are independent given the fields, so a multi-GPU run replicates
the grids and frames on every GPU and splits the particles: no collective on
the data path.  ``shard`` gives each rank a contiguous block of the global
particle index range; the rank's context gets ``set_id_base(start)`` so the
Philox noise of every particle is keyed by its global id and the split run
reproduces a single-GPU run exactly.  ``gather`` collects the ranks' columns
on rank 0 in global order (torch.distributed, any backend).
"""
from __future__ import annotations

from typing import Dict, Tuple

import numpy as np

from . import synth


def shard(n_total: int, rank: int, world: int) -> Tuple[int, int]:
    """(start, count) of rank's block of n_total particles."""
    base, rem = divmod(n_total, world)
    start = rank * base + min(rank, rem)
    count = base + (1 if rank < rem else 0)
    return start, count


def shard_release(rel: synth.Release, rank: int, world: int) -> Tuple[synth.Release, int]:
    n = rel.z.shape[0]
    start, count = shard(n, rank, world)
    sl = slice(start, start + count)
    return synth.Release(ipos=rel.ipos[:, sl].copy(), jpos=rel.jpos[:, sl].copy(), z=rel.z[sl].copy(),
                         dob=rel.dob[sl].copy()), start


def gather(local: Dict[str, np.ndarray], world: int) -> Dict[str, np.ndarray]:
    """Concatenate every rank's columns on all ranks, in rank order."""
    import torch.distributed as dist
    objs = [None] * world
    dist.all_gather_object(objs, local)
    return {k: np.concatenate([o[k] for o in objs]) for k in local}
