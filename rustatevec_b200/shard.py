"""Sharding independent circuits over GPUs (one process per GPU).

A batch of circuits has no data exchange between circuits, so ranks split the circuits and run
their share with no collective on the data path; only the results are gathered on the host. The
split balances estimated cost (sum over gates of 2^n, the amplitudes each gate touches) with the
longest-processing-time rule: circuits in decreasing cost, each to the least-loaded rank.
"""
from __future__ import annotations

import heapq


def circuit_cost(circuit) -> float:
    """Estimated work of one circuit: 2^n amplitudes per gate (at least one gate)."""
    return float(1 << circuit.n_qubits()) * max(1, len(circuit))


def lpt_partition(costs, world: int) -> list:
    """Indices of ``costs`` for each of ``world`` ranks (each list ascending), balanced by LPT."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    parts = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(p) for p in parts]


def execute_batch_sharded(run_share, circuits, world: int, rank: int, group=None):
    """Run this rank's share of ``circuits`` with ``run_share(list_of_circuits) -> (z0, probs)`` and
    gather every circuit's <Z_0> on every rank, in the input order. Probabilities stay on the rank
    that computed them: returns ``(z0_all, my_indices, my_probs)``."""
    parts = lpt_partition([circuit_cost(c) for c in circuits], world)
    mine = parts[rank]
    z0, probs = run_share([circuits[i] for i in mine]) if mine else ([], [])
    pairs = list(zip(mine, [float(x) for x in z0]))
    if world > 1:
        import torch.distributed as dist
        gathered = [None] * world
        dist.all_gather_object(gathered, pairs, group=group)
    else:
        gathered = [pairs]
    z_all = [0.0] * len(circuits)
    for part in gathered:
        for i, z in part:
            z_all[i] = z
    return z_all, mine, probs
