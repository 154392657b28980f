"""Multi-rank host logic on the CPU: gloo, world size 2, one process per rank.

Each rank computes its particle range from the same costs (ranges must tile
[0, n) with balanced cost), integrates nothing, and exercises the reductions
the benchmark and the sharded adjoint use: max of the timings, sum of the
step counts, and the sum of per-rank potential-parameter gradients.
"""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from astrodrift_b200.sharding import balanced_ranges, orbit_cost


def test_balanced_ranges_tile_and_balance():
    rng = np.random.default_rng(0)
    costs = np.exp(rng.uniform(0, 8, 100_000))  # three decades of spread
    for world in (1, 2, 3, 8):
        ranges = balanced_ranges(costs, world)
        assert ranges[0][0] == 0 and ranges[-1][1] == len(costs)
        assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
        sums = np.array([costs[a:b].sum() for a, b in ranges])
        assert sums.max() <= costs.sum() / world + costs.max() + 1e-9


def test_balanced_ranges_small_and_degenerate():
    ranges = balanced_ranges(np.ones(3), 5)  # more ranks than particles: some ranges are empty
    assert ranges[0][0] == 0 and ranges[-1][1] == 3
    assert all(a[1] == b[0] and a[0] <= a[1] for a, b in zip(ranges, ranges[1:]))
    assert balanced_ranges(np.array([]), 2) == [(0, 0), (0, 0)]
    with pytest.raises(ValueError):
        balanced_ranges(np.ones(3), 0)


def test_orbit_cost_counts_dynamical_times():
    # circular Kepler orbit at r = 1: |a| / r = 1 and (v / r)^2 = 1, so the rate is sqrt(2)
    y0 = np.array([[1.0, 0, 0, 0, 1.0, 0]])
    c = orbit_cost(y0, 2 * np.pi, np.array([[-1.0, 0, 0]]))
    assert abs(c[0] - 2 * np.pi * np.sqrt(2.0)) < 1e-12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, queue):
    import datetime

    import torch
    import torch.distributed as dist

    from astrodrift_b200.sharding import reduce_max, reduce_sum, sum_param_grads

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng = np.random.default_rng(1)  # same costs on every rank
        costs = np.exp(rng.uniform(0, 6, 4096))
        lo, hi = balanced_ranges(costs, world)[rank]
        t = reduce_max(0.5 + rank, dist)
        steps = reduce_sum(float(costs[lo:hi].sum()), dist)
        g = torch.full((6,), float(rank + 1), dtype=torch.float64)
        sum_param_grads(g, dist)
        queue.put((rank, lo, hi, t, steps, g.tolist()))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    costs = np.exp(np.random.default_rng(1).uniform(0, 6, 4096))
    (_, lo0, hi0, t0, s0, g0), (_, lo1, hi1, t1, s1, g1) = results
    assert lo0 == 0 and hi0 == lo1 and hi1 == 4096
    assert t0 == t1 == 1.5
    assert abs(s0 - costs.sum()) < 1e-6 * costs.sum() and s0 == s1
    assert g0 == g1 == [3.0] * 6
