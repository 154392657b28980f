"""One process per GPU: particle shards and the few reductions between ranks.

Particles are independent, so the forward integration needs no collective:
each rank integrates a contiguous range of the particles into its own HBM.
Ranges are balanced by estimated cost (the number of dynamical times in a
particle's span, the quantity the ordered schedule ranks by), so that ranks
finish together on uneven workloads such as per-particle end times spanning
two decades.  What crosses ranks is small: the timing (max), step counts
(sum) and, for the adjoint, the potential-parameter gradients (a sum of at
most DRIFT_ADJOINT_MAX_PARAMS doubles).  The helpers take any initialised
torch.distributed process group: NCCL on GPUs, gloo in the CPU tests.
"""

from __future__ import annotations

import numpy as np


def orbit_cost(y0: np.ndarray, span, accel: np.ndarray) -> np.ndarray:
    """Dynamical times in each particle's span: |span| sqrt(|a| / r + (v / r)^2).

    y0 (n, 6); span scalar or (n,); accel (n, 3) the force at the initial
    positions (drift_force)."""
    r2 = np.maximum((y0[:, :3] ** 2).sum(1), 1e-300)
    v2 = (y0[:, 3:] ** 2).sum(1)
    a = np.sqrt((accel ** 2).sum(1))
    cost = np.abs(np.asarray(span, dtype=np.float64)) * np.sqrt(a / np.sqrt(r2) + v2 / r2)
    return np.where(np.isfinite(cost) & (cost > 0), cost, 1.0)


def balanced_ranges(costs: np.ndarray, world: int) -> list[tuple[int, int]]:
    """Split [0, n) into `world` contiguous ranges with near-equal cost sums.

    Rank r takes [cut_r, cut_{r+1}) where cut_r is the first index whose
    prefix cost reaches r / world of the total.  Every rank computes the same
    cuts from the same costs, so no communication is needed."""
    costs = np.asarray(costs, dtype=np.float64)
    n = len(costs)
    if world < 1:
        raise ValueError("world must be >= 1")
    prefix = np.concatenate([[0.0], np.cumsum(costs)])
    total = prefix[-1]
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(prefix, total * r / world, side="left")))
    cuts.append(n)
    cuts = np.maximum.accumulate(np.clip(cuts, 0, n))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def reduce_max(value: float, dist, device=None) -> float:
    """Max of a scalar over the ranks of the default group."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(value: float, dist, device=None) -> float:
    """Sum of a scalar over the ranks of the default group."""
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def sum_param_grads(grad, dist):
    """In-place sum over ranks of a potential-parameter gradient tensor (the
    only exchange the sharded adjoint needs); returns it."""
    dist.all_reduce(grad, op=dist.ReduceOp.SUM)
    return grad
