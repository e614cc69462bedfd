"""Parameter sets across GPUs.

DENSE's sets are independent simulations (run_simulation loops over them,
run_simulation.hpp:152-157), so a multi-GPU run partitions them with no
exchange during stepping: each rank (one process per GPU, torch.distributed)
builds a batch from its share and runs it; the per-set outputs are gathered
once at the end.
"""

import heapq

import numpy as np


def set_cost(num_cells, duration, interval, step_size):
    """Cell-steps of one set: cells x chunks x (int)(interval / dt)."""
    chunks = int(np.ceil(duration / interval))
    return num_cells * chunks * int(interval / step_size)


def shard(costs, world):
    """Longest-processing-time assignment of set indices to `world` ranks:
    sets in decreasing cost, each to the currently lightest rank.  Returns
    one ascending index list per rank."""
    heap = [(0, r) for r in range(world)]
    out = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda k: (-costs[k], k)):
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return [sorted(x) for x in out]


def gather_rows(local_rows, local_index, total, group=None):
    """Collect per-set result rows from every rank into one [total, ...]
    array on every rank (torch.distributed all_gather_object; a few values
    per set, once per run)."""
    import torch.distributed as dist
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, (list(local_index), np.asarray(local_rows)), group=group)
    first = next(p[1] for p in parts if len(p[0]))
    out = np.zeros((total,) + first.shape[1:], first.dtype)
    for idx, rows in parts:
        if len(idx):
            out[np.asarray(idx)] = rows
    return out
