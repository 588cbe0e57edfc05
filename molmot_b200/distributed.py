"""Multi-GPU sharding of the rate-equation workloads (one process per GPU).

Every workload of this path is a set of independent units -- parameter sets
of a force map, molecules of an uneven batch, particles of an ensemble -- so
ranks split the units into contiguous blocks and compute them with no
collective on the data path.  Collectives appear only where a caller wants
all results everywhere (``all_gather`` of a map) or an ensemble statistic
(``all_reduce`` of a few sums); with the NCCL backend they run over
NVLink/NVSwitch, with gloo on CPU tensors for tests.
"""
from __future__ import annotations

from typing import Callable, Optional, Tuple

import torch
import torch.distributed as dist


def world() -> Tuple[int, int]:
    """(rank, world_size); (0, 1) without an initialised process group."""
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(), dist.get_world_size()
    return 0, 1


def shard(n_units: int, rank: int, world_size: int) -> Tuple[int, int]:
    """Contiguous block [lo, hi) of n_units for rank; sizes differ by at most one."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError(f"bad rank {rank} / world size {world_size}")
    base, extra = divmod(n_units, world_size)
    lo = rank * base + min(rank, extra)
    hi = lo + base + (1 if rank < extra else 0)
    return lo, hi


def sharded_apply(n_units: int, compute: Callable[[int, int], torch.Tensor], gather: bool = False,
                  group=None) -> torch.Tensor:
    """Run compute(lo, hi) on this rank's block of units.  With gather=True the
    per-unit results (leading dimension = units) of every rank are
    concatenated in unit order on every rank (all_gather of padded blocks)."""
    rank, ws = world()
    lo, hi = shard(n_units, rank, ws)
    out = compute(lo, hi)
    if not gather or ws == 1:
        return out
    base, extra = divmod(n_units, ws)
    maxn = base + (1 if extra else 0)
    pad = torch.zeros((maxn,) + tuple(out.shape[1:]), dtype=out.dtype, device=out.device)
    pad[: out.shape[0]] = out
    parts = [torch.empty_like(pad) for _ in range(ws)]
    dist.all_gather(parts, pad, group=group)
    blocks = []
    for r in range(ws):
        a, b = shard(n_units, r, ws)
        blocks.append(parts[r][: b - a])
    return torch.cat(blocks, 0)


def ensemble_mean(values: torch.Tensor, mask: Optional[torch.Tensor] = None, group=None) -> float:
    """Mean of per-particle values over all ranks' particles (one all_reduce of
    a sum and a count)."""
    if mask is None:
        mask = torch.ones_like(values, dtype=torch.bool)
    acc = torch.stack([(values * mask).sum().to(torch.float64),
                       mask.sum().to(torch.float64)])
    _, ws = world()
    if ws > 1:
        dist.all_reduce(acc, op=dist.ReduceOp.SUM, group=group)
    return float(acc[0] / acc[1]) if acc[1] > 0 else float("nan")


def sharded_force_maps(mol, kdir, freq, pol, s0, bgrad, v, z, precision="fp32", gather=False,
                       group=None):
    """Force maps of n_sets parameter sets (v x z grids), sets sharded over
    ranks, each rank on its own GPU.  Returns this rank's block
    [sets_local, nv, nz], or with gather=True all sets on every rank."""
    from .engine import BeamSets, force_batch, pack_for
    import numpy as np
    kdir = np.atleast_2d(kdir)

    def compute(lo, hi):
        bs = BeamSets(kdir[lo:hi], np.asarray(freq)[lo:hi], np.asarray(pol)[lo:hi],
                      np.asarray(s0)[lo:hi], np.asarray(bgrad)[lo:hi])
        return force_batch(pack_for(mol), bs, v, z, grid=True, precision=precision,
                           want_pop=False, want_R=False, want_status=False)["F"]

    return sharded_apply(kdir.shape[0], compute, gather, group)
