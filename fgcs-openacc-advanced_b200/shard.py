"""Work split across ranks (one process per GPU) for the two workloads that
partition: the instances of a batch (fold3d_solve_batch) and the sources of a
tomography survey (one forward solve and one adjoint each).  Both are sets of
independent solves, so the only collective is the one after them: the sum of
the sources' gradients.  A single solve does not split (every plane step reads
the whole previous plane) and runs as replicas.

partition() is deterministic and needs no communication: every rank computes
the same split from the same cost list and takes its own part.
"""
from __future__ import annotations


def partition(costs, parts):
    """Greedy longest-processing-time split of items with the given costs
    (cells of each instance, or 1 per source) into `parts` parts: items by
    decreasing cost (ties by lower index), each to the part with the smallest
    total so far (ties by lower part number).  Returns `parts` lists of item
    indices, each ascending.  The largest part total is at most
    sum(costs) / parts + max(costs)."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    costs = [float(c) for c in costs]
    if any(c < 0 for c in costs):
        raise ValueError("costs must be non-negative")
    load = [0.0] * parts
    out = [[] for _ in range(parts)]
    for i in sorted(range(len(costs)), key=lambda q: (-costs[q], q)):
        p = min(range(parts), key=lambda q: (load[q], q))
        out[p].append(i)
        load[p] += costs[i]
    return [sorted(o) for o in out]


def rank_and_world(dist=None):
    """(rank, world size) of the joined process group, or (0, 1)."""
    if dist is None or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(), dist.get_world_size()


def sum_over_ranks_(tensors, dist=None):
    """In-place sum of each tensor over all ranks (one all-reduce per tensor,
    in list order, the same on every rank); identity for a single process.
    Returns the list."""
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        for t in tensors:
            dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return tensors
