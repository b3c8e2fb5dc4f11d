"""Sharding of independent cases across ranks (one process per GPU).

Only the batched-serving path shards: its cases are independent, so they are split across
ranks by the greedy longest-processing-time rule on an estimated cost and each rank solves
its share alone; there is no data-path collective, only host-side reductions of timings and
metrics (torch.distributed with NCCL on GPUs, gloo on CPU).
"""
import numpy as np


def case_cost(n_elements, order, n_eqs=4, dim=2):
    """Estimated cost of one case: unknowns x block size (the block-Jacobi factor and the
    element Jacobian grow with the square of the element block)."""
    nb = order * (order + 1) // 2 if dim == 2 else order * (order + 1) * (order + 2) // 6
    nc = nb * n_eqs
    return float(n_elements) * nc * nc


def lpt_partition(costs, n_parts):
    """Greedy longest-processing-time assignment: cases by decreasing cost (ties by index),
    each to the currently least-loaded part (ties by part index).  Returns a list of index
    lists, one per part, each in increasing case order."""
    costs = np.asarray(costs, dtype=np.float64)
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = np.zeros(n_parts)
    parts = [[] for _ in range(n_parts)]
    for i in order:
        p = int(np.argmin(load))
        parts[p].append(i)
        load[p] += costs[i]
    return [sorted(p) for p in parts]


def max_over_ranks(value, device=None):
    """max of a float over all ranks (the value itself without an initialised process group)"""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_metrics(obj):
    """all ranks' objects as a list indexed by rank ([obj] without a process group)"""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return [obj]
    out = [None] * dist.get_world_size()
    dist.all_gather_object(out, obj)
    return out
