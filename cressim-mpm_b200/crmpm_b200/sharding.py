"""Scene sharding of a batch across GPUs (one process per GPU).

Scenes are independent (no exchange step), so a batch splits by scene: each rank builds a
``DeviceBatch`` of its own scenes and no collective touches the particle data.  Scenes go to ranks
by greedy largest-first balance of particle counts, which keeps the slowest rank within one
scene's worth of work of the mean.
"""
from __future__ import annotations


def shard_scenes(counts, world: int) -> list[list[int]]:
    """Scene indices per rank: largest scene first onto the least-loaded rank (ties: lower rank,
    then lower scene index), each rank's list in ascending scene order.  Deterministic, so every
    rank computes the same assignment without communicating."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(counts)), key=lambda s: (-int(counts[s]), s))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for s in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(s)
        load[r] += int(counts[s])
    return [sorted(o) for o in out]


def shard_loads(counts, shards) -> list[int]:
    return [sum(int(counts[s]) for s in sh) for sh in shards]
