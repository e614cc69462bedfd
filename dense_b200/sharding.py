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


def _engine_run(model, sets, step_size, analysis_interval, analyses, precision, device, with_state):
    """One engine batch of `sets` on `device` to the end of every horizon:
    per set its status word, Oscillation amplitudes and periods (per
    Oscillation analysis) and, with `with_state`, its lag-0 state."""
    from . import engine as E
    b = E.Batch(model, sets, step_size, analysis_interval, analyses,
                precision=E.FP64 if precision is None else precision, device=device)
    try:
        b.run()
        b.sync()
        out = {"status": b.status()}
        for ai, a in enumerate(b.analyses):
            if a.kind == E.OSCILLATION:
                out["amps_%d" % ai], out["pers_%d" % ai] = b.oscillation_all(ai)
        if with_state:
            out["state"] = [b.state(i) for i in range(len(sets))]
        return out
    finally:
        b.close()


def simulate_sharded(model, sets, step_size, analysis_interval, analyses=(), precision=None, group=None,
                     device=None, with_state=False, run_batch=None):
    """Runs `sets` over the ranks of `group` (one process per GPU, the
    default group when torch.distributed is initialized, else this process
    alone): each rank takes its cost-balanced share (shard of set_cost),
    runs it as one batch on its GPU with no exchange during stepping, and
    the per-set results are gathered once, on every rank.

    Returns {"status": [n] int32, "amps_<a>"/"pers_<a>": [n][species][cells]
    for each Oscillation analysis a, "state": [n] list of [species][cells]
    (with `with_state`), "shares": the set indices of every rank}.
    `run_batch` has the signature of the engine runner (the default) and
    returns the same keys for its list of sets."""
    import os
    import torch.distributed as dist
    on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if on else 0
    world = dist.get_world_size(group) if on else 1
    if device is None:
        device = int(os.environ.get("LOCAL_RANK", "0"))
    costs = [set_cost(s.num_cells, s.duration, analysis_interval, step_size) for s in sets]
    shares = shard(costs, world)
    mine = shares[rank]
    run = run_batch or _engine_run
    local = run(model, [sets[i] for i in mine], step_size, analysis_interval, list(analyses), precision, device,
                with_state) if mine else {}
    # one gather of the per-set rows (objects: the sets' cell counts differ)
    rows = [(i, {k: (v[j] if k == "state" else np.asarray(v)[j]) for k, v in local.items()})
            for j, i in enumerate(mine)]
    parts = [None] * world
    if on:
        if dist.get_backend(group) == "nccl":
            import torch
            torch.cuda.set_device(device)  # NCCL stages the objects on the current device
        dist.all_gather_object(parts, rows, group=group)
    else:
        parts = [rows]
    by_set = dict(r for p in parts for r in p)
    n = len(sets)
    keys = sorted({k for r in by_set.values() for k in r})
    out = {"shares": shares}
    for k in keys:
        vals = [by_set[i][k] for i in range(n)]
        out[k] = vals if k == "state" else np.stack(vals)
    return out
