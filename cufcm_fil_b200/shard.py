"""Sharding a batch of independent wall arrays over ranks (one process per GPU).

The reference's sweep drivers (pyfile/find_periodic, pyfile/bisection) run many
independent simulations; the reference itself only splits one array's targets
over GPUs, with host-staged replicas (rpy_mobility_solver.cu:58-87).  Here the
unit of work is a whole array: the arrays share nothing, so each rank steps
its own bin of arrays as one batch (cf_batch) and the data path has no
collective at all.  Only the per-array results are gathered at the end, over
whatever process group the caller set up (NCCL or gloo).

  array_cost(n_fil, nseg)     the pair-product work of one array per GMRES iteration
  bin_by_cost(costs, world)   longest-processing-time binning, deterministic
  gather_to_root(obj, world)  per-rank results -> list on rank 0 (None elsewhere)
"""
from __future__ import annotations


def array_cost(n_fil: int, nseg: int) -> int:
    """Directed segment pairs of one matvec: the O(N^2) pair product dominates a step."""
    n = int(n_fil) * int(nseg)
    return n * n


def bin_by_cost(costs, world: int) -> list[list[int]]:
    """Assigns array indices to `world` bins, heaviest first onto the least-loaded bin (ties: lowest bin, then
    lowest index), so every rank computes the same assignment without communicating.  Each bin is returned in
    ascending index order."""
    world = int(world)
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    load = [0] * world
    bins: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        bins[r].append(i)
        load[r] += int(costs[i])
    return [sorted(b) for b in bins]


def imbalance(costs, bins) -> float:
    """Largest bin cost over the mean bin cost (1.0 = perfect balance)."""
    loads = [sum(int(costs[i]) for i in b) for b in bins]
    mean = sum(loads) / max(1, len(loads))
    return max(loads) / mean if mean else 1.0


def gather_to_root(obj, world: int):
    """Every rank's `obj` as a list on rank 0 (rank order); None on the other ranks.  A no-op list at world 1."""
    if int(world) == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * int(world) if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out
