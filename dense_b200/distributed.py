"""Host-side pieces of the multi-GPU surrogate search (one process per GPU,
torch.distributed: NCCL on GPUs, gloo in the CPU tests).

* Candidates are drawn in fixed chunks, each from its own seeded stream, so
  any rank can draw any range or any single candidate without drawing the
  rest (`candidate_range`, `candidates_at`).
* Surrogate screening keeps the global top k of the scores: every rank
  sends its local top k, every rank merges the same way (`global_top`).
* Data-parallel surrogate training averages the gradients of all ranks in
  one flat all-reduce per step (`average_`).
"""

import numpy as np

CHUNK = 1 << 16


def shard_range(n, rank, world):
    """Contiguous [lo, hi) share of n items for `rank` of `world`."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _chunk(seed, c, draw):
    return draw(np.random.Generator(np.random.PCG64([int(seed), int(c)])), CHUNK)


def candidate_range(lo, hi, seed, draw):
    """Rows lo..hi-1 of the candidate sequence; `draw(rng, m)` draws m rows."""
    if hi <= lo:
        return draw(np.random.Generator(np.random.PCG64(0)), 0)
    parts = []
    for c in range(lo // CHUNK, (hi - 1) // CHUNK + 1):
        rows = _chunk(seed, c, draw)
        a, b = max(lo, c * CHUNK) - c * CHUNK, min(hi, (c + 1) * CHUNK) - c * CHUNK
        parts.append(rows[a:b])
    return np.concatenate(parts)


def candidates_at(indices, seed, draw):
    """The candidates with the given global indices (any order)."""
    indices = np.asarray(indices, np.int64)
    out = None
    for c in np.unique(indices // CHUNK):
        rows = _chunk(seed, c, draw)
        sel = np.nonzero(indices // CHUNK == c)[0]
        if out is None:
            out = np.empty((len(indices),) + rows.shape[1:], rows.dtype)
        out[sel] = rows[indices[sel] - c * CHUNK]
    if out is None:
        out = draw(np.random.Generator(np.random.PCG64(0)), 0)
    return out


def _order(scores, indices):
    """Descending score, ascending index among equal scores (NaN last)."""
    s = np.where(np.isnan(scores), -np.inf, scores)
    return np.lexsort((indices, -s))


def local_top(scores, indices, k):
    """The k best (score, index) pairs in _order's order.  With k below the
    count, a partition finds the k-th best score first and only the
    candidates at or above it (ties included) are sorted."""
    scores = np.asarray(scores, np.float64)
    indices = np.asarray(indices, np.int64)
    n = scores.size
    if 0 < k < n:
        s = np.where(np.isnan(scores), -np.inf, scores)
        kth = np.partition(s, n - k)[n - k]
        keep = np.nonzero(s >= kth)[0]
        o = keep[_order(scores[keep], indices[keep])[:k]]
    else:
        o = _order(scores, indices)[:max(k, 0)]
    return scores[o], indices[o]


def global_top(scores, indices, k, group=None):
    """Global indices of the k best scores over all ranks, best first; the
    same array on every rank.  Without a process group: the local top k."""
    s, i = local_top(scores, indices, k)
    import torch.distributed as dist
    if group is None and not (dist.is_available() and dist.is_initialized()):
        return i
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, (s, i), group=group)
    s = np.concatenate([p[0] for p in parts])
    i = np.concatenate([p[1] for p in parts])
    return i[_order(s, i)[:k]]


def average_(tensors, group=None):
    """In-place mean of the tensors over all ranks: one all-reduce of their
    concatenation."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return
    world = dist.get_world_size(group)
    if world == 1:
        return
    flat = torch.cat([t.reshape(-1) for t in tensors])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    flat /= world
    o = 0
    for t in tensors:
        n = t.numel()
        t.copy_(flat[o:o + n].view_as(t))
        o += n
