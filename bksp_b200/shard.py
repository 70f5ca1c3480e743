"""Partition of a batch of independent systems over GPUs.

The batched workload is the one part of the solver path that shards: its
systems are independent, so each rank solves a subset and no data crosses
between GPUs (only the timings are reduced).  The split balances the work,
taken as the stored entries of each system (one SpMV and the vector updates
scale with it), by the longest-processing-time rule: systems in decreasing
size order, each to the currently lightest rank.  Deterministic, so every
rank computes the same partition without communication.
"""


def partition(weights, parts):
    """Indices of the systems of each of `parts` shares (lists, each in
    increasing index order)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-weights[i], i))
    load = [0.0] * parts
    shares = [[] for _ in range(parts)]
    for i in order:
        r = min(range(parts), key=lambda p: (load[p], p))
        shares[r].append(i)
        load[r] += weights[i]
    return [sorted(s) for s in shares]


def my_share(weights, world, rank):
    """The systems rank `rank` of `world` solves."""
    if not 0 <= rank < world:
        raise ValueError("rank out of range")
    return partition(weights, world)[rank]
