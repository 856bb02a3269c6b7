"""Splitting independent search units across ranks.

Units (target chunk x query x strand) are independent: every reference
search() call starts from a fresh DiagHash (src/seed_search.rs:58) and the
driver only concatenates results (src/driver.rs:362-391).  So N GPUs take
disjoint shares of the units with no collective on the data path.
"""
from __future__ import annotations


def shard_units(n_units: int, rank: int, world: int, weights=None) -> list[int]:
    """Indices of the units rank `rank` of `world` runs.

    With weights (e.g. query lengths) units go greedily, heaviest first, to the
    least-loaded rank; ties go to the lower rank, so every rank computes the
    same assignment without communicating."""
    if world <= 1:
        return list(range(n_units))
    if weights is None:
        return list(range(rank, n_units, world))
    order = sorted(range(n_units), key=lambda i: (-weights[i], i))
    load = [0.0] * world
    owner = [0] * n_units
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        owner[i] = r
        load[r] += weights[i]
    return [i for i in range(n_units) if owner[i] == rank]
