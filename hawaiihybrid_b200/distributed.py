"""Multi-GPU form of the correlation pass: one process per GPU.

Trajectories are independent, so each rank draws its own from its own MT19937
seed, as the reference gives each MPI rank its own seed (per-rank seed table of
examples/correlation_he_ar.cpp:133-137).  The one exchange step is the
reference's rank-0 gather of C(t) (src/hawaii.c:3015-3038), here a single
all-reduce (SUM) of C(t) and the trajectory count.  With the NCCL backend it
runs over NVLink on device buffers; with gloo (tests) on host tensors.
"""
from __future__ import annotations

from typing import Callable, Optional

import numpy as np

SEED_STRIDE = 1000


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed of rank `rank`: distinct, non-zero, and base_seed itself on rank 0."""
    return int(base_seed) + SEED_STRIDE * int(rank)


def correlation_iteration_sharded(ms, params, Temperature: float, n_per_rank: int, precision: int,
                                  base_seed: int, group=None,
                                  compute: Optional[Callable] = None, device: Optional[str] = None):
    """One accumulation pass over world_size * n_per_rank trajectories.

    Returns (crln_sum, ntraj, local_stats) with crln_sum and ntraj summed over
    ranks.  `compute(ms, params, T, n, precision, seed)` defaults to the device
    call hawaii.correlation_iteration."""
    import torch
    import torch.distributed as dist

    if compute is None:
        from .hawaii import correlation_iteration as compute
    rank = dist.get_rank(group)
    crln, ntraj, st = compute(ms, params, Temperature, n_per_rank, precision, rank_seed(base_seed, rank))
    buf = torch.from_numpy(np.append(np.asarray(crln, dtype=np.float64), float(ntraj)))
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return out[:-1], float(out[-1]), st
