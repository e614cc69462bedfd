"""Host logic of the multi-GPU surrogate search on CPU: candidate chunks,
the global top-k merge across two gloo ranks, and the gradient average."""

import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from dense_b200 import distributed as D


def _draw(rng, m):
    return rng.uniform(size=(m, 3))


def test_candidate_range_and_at_agree():
    n = 3 * D.CHUNK + 123
    full = D.candidate_range(0, n, 7, _draw)
    assert full.shape == (n, 3)
    assert np.array_equal(D.candidate_range(D.CHUNK - 5, 2 * D.CHUNK + 9, 7, _draw),
                          full[D.CHUNK - 5:2 * D.CHUNK + 9])
    idx = np.array([n - 1, 0, D.CHUNK, 17, 2 * D.CHUNK + 1])
    assert np.array_equal(D.candidates_at(idx, 7, _draw), full[idx])
    parts = [D.shard_range(n, r, 3) for r in range(3)]
    assert parts[0][0] == 0 and parts[-1][1] == n
    assert all(parts[r][1] == parts[r + 1][0] for r in range(2))


def test_local_top_orders_ties_and_nan():
    s = np.array([1.0, np.nan, 3.0, 3.0, 2.0])
    i = np.array([10, 11, 12, 9, 13])
    _, top = D.local_top(s, i, 4)
    assert list(top) == [9, 12, 13, 10]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.Generator(np.random.PCG64(3))
    n = 1000
    scores = np.round(rng.normal(size=n), 2)  # many ties
    lo, hi = D.shard_range(n, rank, world)
    top = D.global_top(scores[lo:hi], np.arange(lo, hi), 37)
    g = [torch.full((4,), float(rank + 1)), torch.full((2, 3), 10.0 * (rank + 1))]
    D.average_(g)
    out[rank] = (top.tolist(), g[0].tolist(), g[1].reshape(-1).tolist())
    dist.destroy_process_group()


def test_two_rank_global_top_and_average():
    mp_ctx = mp.get_context("spawn")
    with mp_ctx.Manager() as m:
        out = m.dict()
        port = 29613
        procs = [mp_ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    rng = np.random.Generator(np.random.PCG64(3))
    scores = np.round(rng.normal(size=1000), 2)
    _, want = D.local_top(scores, np.arange(1000), 37)
    for r in range(2):
        top, g0, g1 = res[r]
        assert top == want.tolist()
        assert g0 == [1.5] * 4 and g1 == [15.0] * 6


def test_local_top_partition_path_equals_a_full_sort():
    """local_top's partition prefilter returns exactly the first k of the
    full order (descending score, ascending index among ties, NaN last)."""
    from dense_b200.distributed import _order, local_top
    rng = np.random.Generator(np.random.PCG64(12))
    for n, k in ((1000, 10), (1000, 999), (1000, 1000), (1000, 1500), (50, 0), (2000, 300)):
        s = rng.integers(0, 20, size=n).astype(np.float64)   # many ties
        s[rng.choice(n, size=n // 10, replace=False)] = np.nan
        idx = rng.permutation(n).astype(np.int64) + 7
        full = _order(s, idx)[:k]
        got_s, got_i = local_top(s, idx, k)
        assert np.array_equal(got_i, idx[full])
        assert np.array_equal(got_s, s[full], equal_nan=True)
