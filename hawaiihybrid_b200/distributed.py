"""Multi-GPU form of the correlation pass and of the moment integrals: one process per GPU.

Trajectories are independent, so each rank draws its own from its own MT19937
seed, as the reference gives each MPI rank its own seed (per-rank seed table of
examples/correlation_he_ar.cpp:133-137).  The one exchange step is the
reference's rank-0 gather of C(t) (src/hawaii.c:3015-3038), here a single
all-reduce (SUM) of C(t) and the trajectory count.  With the NCCL backend it
runs over NVLink on device buffers; with gloo (tests) on host tensors.

The moment integrals shard the same way as the reference's mpi_calculate_M0 /
mpi_calculate_M2 (src/hawaii.c:1620-1738, 1740-1856), where every rank integrates
its own points and rank 0 sums the per-rank (m, q) pairs: here rank r evaluates
the Philox counters [r n_per_rank, (r + 1) n_per_rank) of one stream, and one
all-reduce (SUM) of the per-temperature (sum w, sum w^2) gives the moments of all
world_size * n_per_rank samples, the same samples a single rank would draw.
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


def moment_sharded(ms, params, temperatures, n_per_rank: int, seed: int, moment: int = 0, precision: int = 0,
                   group=None, compute: Optional[Callable] = None, device: Optional[str] = None):
    """M0 (moment 0) or M2 (moment 2) over world_size * n_per_rank samples.

    Returns (m, err) at every temperature, equal on all ranks.  `compute(ms, params, T,
    n, offset, seed, moment, precision)` returns the per-temperature (sum w, sum w^2)
    over the samples [offset, offset + n); it defaults to the device call
    hawaii.moment_sums."""
    import torch
    import torch.distributed as dist

    from .hawaii import moment_from_sums, moment_scale
    if compute is None:
        from .hawaii import moment_sums

        def compute(ms_, p_, T_, n_, off_, seed_, mom_, prec_):
            return moment_sums(ms_, p_, T_, n_, sample_offset=off_, seed=seed_, moment=mom_, precision=prec_)
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    T = np.asarray(temperatures, dtype=np.float64)
    sw, sw2 = compute(ms, params, T, n_per_rank, rank * n_per_rank, seed, moment, precision)
    buf = torch.from_numpy(np.concatenate([np.asarray(sw, dtype=np.float64), np.asarray(sw2, dtype=np.float64)]))
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return moment_from_sums(out[:T.size], out[T.size:], world * n_per_rank, moment_scale(params, moment))
