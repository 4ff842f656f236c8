"""Sharding of independent transforms across ranks (one process per GPU).

The NUFFT path partitions into independent units — the instances of a batch
and the transforms of an instance — with no exchange between them, so several
GPUs share a workload by splitting the units, with no collective on the data
path.  ``assign`` balances units by weight (for example points x transforms)
with the longest-processing-time rule: units in decreasing weight, each to
the rank with the least weight so far (ties to the lower rank), which is
deterministic, so every rank computes the same assignment without
communication.  ``local_units`` is the part of one rank.
"""

__all__ = ["assign", "local_units"]


def assign(weights, world):
    """Unit indices per rank: a list of ``world`` sorted lists."""
    if world < 1:
        raise ValueError("world must be >= 1")
    w = [float(x) for x in weights]
    if any(x < 0 for x in w):
        raise ValueError("weights must be non-negative")
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += w[i]
    return [sorted(p) for p in parts]


def local_units(weights, rank, world):
    """Unit indices of ``rank``."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return assign(weights, world)[rank]
