"""Sharding of independent worlds across ranks (one process per GPU).

Worlds never interact, so the batched workload partitions with no data
exchange: rank r builds and steps its own worlds, seeded from
`rank_seed(base, r)`, with body counts drawn by the scene generator's
log-uniform size rule.  Only timing and results cross ranks.
"""
from __future__ import annotations

RANK_STRIDE = 1_000_003


def rank_seed(base_seed: int, rank: int) -> int:
    return base_seed + RANK_STRIDE * rank


def shard_sizes(lib, seed: int, count: int, lo: int, hi: int) -> list[int]:
    """Dynamic body counts of a rank's `count` worlds (log-uniform [lo, hi])."""
    return [int(lib.m3s_uneven_size(seed, i, lo, hi)) for i in range(count)]


def world_seeds(seed: int, count: int) -> list[int]:
    return [seed + i for i in range(count)]
