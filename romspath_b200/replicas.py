"""Particle sharding for runs on several GPUs (one process per GPU).

Particles are independent given the fields, so a multi-GPU run replicates
the grids and frames on every GPU and splits the particles: no collective on
the data path.  ``shard`` gives each rank a contiguous block of the global
particle index range; the rank's context gets ``set_id_base(start)`` so the
Philox noise of every particle is keyed by its global id and the split run
reproduces a single-GPU run exactly.  ``gather`` collects the ranks' columns
on rank 0 in global order (torch.distributed, any backend).

The two quantities that do sum over particles are reduced at output or
loss time, never per step: the adjoint's dL/dkappa (each rank's
rp_backward sums its own particles' contributions) and the concentration
histograms of the particles (``global_profile``).  Per-particle
gradients stay on their rank.
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


def _reduce_device():
    import torch
    import torch.distributed as dist
    if dist.get_backend() == "nccl":
        return torch.device("cuda", torch.cuda.current_device())
    return torch.device("cpu")


def allreduce_sum(x):
    """Sum of x (a number or an array) over all ranks: one all_reduce of a
    float64 tensor (on the current GPU under NCCL)."""
    import torch
    import torch.distributed as dist
    a = np.asarray(x, dtype=np.float64)
    t = torch.from_numpy(a.reshape(-1).copy()).to(_reduce_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    out = t.cpu().numpy().reshape(a.shape)
    return float(out) if out.ndim == 0 else out


def kappa_gradient(local_dl_dkappa: float) -> float:
    """dL/dkappa of the whole particle set from each rank's rp_backward
    value (the loss is a sum over particles, each particle's trajectory
    depends on kappa alone, so the gradient is the sum of the shards')."""
    return allreduce_sum(float(local_dl_dkappa))


MOVED_STATUS = (1.0, float(np.float32(1.1)), float(np.float32(1.2)))


def column_profile(state: Dict[str, np.ndarray], bins: int = 20) -> np.ndarray:
    """Counts of this rank's moving particles (status 1, 1.1, 1.2) in
    `bins` equal bins of the water-column fraction (z + h) / (h + zeta)."""
    ok = np.isin(state["status"], MOVED_STATUS)
    h = state["bath"][ok]
    frac = (state["z"][ok] + h) / (h + state["zeta"][ok])
    return np.histogram(frac, bins=bins, range=(0.0, 1.0))[0].astype(np.float64)


def global_profile(state: Dict[str, np.ndarray], bins: int = 20) -> np.ndarray:
    """The vertical concentration profile of all ranks' particles (the
    sum of every rank's ``column_profile``), on every rank."""
    return allreduce_sum(column_profile(state, bins))
