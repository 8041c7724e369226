"""Sharding of independent worlds across ranks (one process per GPU).

Worlds never interact, so a batch partitions with no data exchange on the
step path: every rank receives the same world list, keeps the worlds
`partition` assigns to it, builds and steps only those, and only timing
and results (the worlds' 64-bit hashes) cross ranks.

The partition balances estimated cost, not world count: a world's step
work grows with its bodies and its candidate pairs (the narrowphase, the
contact rows of the solver), so each world is weighed by
`world_cost(bodies, pairs)` and the list is split by the longest-
processing-time rule -- heaviest world first, each to the rank with the
least cost so far (ties to the lower rank).  The result depends only on
the costs and the rank count, so every rank computes the same split
without talking to the others.
"""
from __future__ import annotations

# Candidate pairs per dynamic body when a world's pair count is not known
# yet (settled box stacks and loose spheres carry about two to three).
PAIRS_PER_BODY_ESTIMATE = 3


def shard_sizes(lib, seed: int, count: int, lo: int, hi: int) -> list[int]:
    """Dynamic body counts of `count` seeded worlds (log-uniform [lo, hi])."""
    return [int(lib.m3s_uneven_size(seed, i, lo, hi)) for i in range(count)]


def world_cost(bodies: int, pairs: int | None = None) -> int:
    """Estimated step cost of one world: bodies plus candidate pairs (the
    pair count measured on an earlier step when known, else estimated)."""
    if pairs is None:
        pairs = PAIRS_PER_BODY_ESTIMATE * bodies
    return int(bodies) + int(pairs)


def partition(costs: list[int], ranks: int) -> list[list[int]]:
    """Indices of `costs` per rank, balanced by total cost (greedy
    longest-processing-time; deterministic).  Each rank's list is in
    ascending index order."""
    if ranks <= 0:
        raise ValueError("ranks must be positive")
    load = [0] * ranks
    out: list[list[int]] = [[] for _ in range(ranks)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        r = min(range(ranks), key=lambda q: (load[q], q))
        load[r] += costs[i]
        out[r].append(i)
    return [sorted(x) for x in out]
