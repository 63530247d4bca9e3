"""Multi-process layout of the vertical advance.

Columns are independent within a step, so GITM's domain decomposition
(blocks of lat/lon columns per MPI rank, srcSphereAB/, srcDoc/grid.tex:9-18)
becomes a contiguous split of each member's columns over ranks with no data
exchange.  The one collective the reference has on this path is the time
step: calc_timestep_vertical takes MPI_Allreduce(MIN) of the local CFL step
(calc_timestep.f90:144-145); ``global_dt`` is that reduction over
torch.distributed (NCCL between GPUs, gloo on CPU).
"""
from __future__ import annotations

import dataclasses

import numpy as np


def shard_range(n_cols: int, rank: int, world: int) -> tuple[int, int]:
    """[c0, c1) of the columns rank owns: contiguous, sizes differing by <= 1."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_cols, world)
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


def shard_member(m, rank: int, world: int):
    """The columns [c0, c1) of a synthetic.Member (numpy) as a new Member."""
    c0, c1 = shard_range(m.n_cols, rank, world)
    kw = {}
    for f in dataclasses.fields(m):
        v = getattr(m, f.name)
        if f.name == "n_cols":
            kw[f.name] = c1 - c0
        elif isinstance(v, np.ndarray):
            if f.name in ("altitude", "gravity", "dalt_c", "inv_r") and v.ndim == 1:
                kw[f.name] = v.copy()  # one grid shared by all columns
            else:
                kw[f.name] = np.ascontiguousarray(v[..., c0:c1])
        else:
            kw[f.name] = v
    return type(m)(**kw)


def global_dt(local_dt: float, group=None, device=None) -> float:
    """MPI_Allreduce(MIN) of calc_timestep_vertical over the process group."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([local_dt], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())
