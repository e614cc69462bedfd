"""Multi-GPU host path on CPU: sets shard across two gloo ranks, each rank
simulates its share (the oracle stands in for the engine here), and the
gathered per-set results equal a single-process run."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from dense_b200.sharding import set_cost, shard


def test_shard_partitions_and_balances():
    rng = np.random.Generator(np.random.PCG64(5))
    costs = list(rng.integers(1, 1000, size=257))
    parts = shard(costs, 4)
    assert sorted(i for p in parts for i in p) == list(range(257))
    loads = [sum(costs[i] for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(costs)
    assert shard([5, 5], 4)[2:] == [[], []]


def test_set_cost():
    assert set_cost(200, 1200.0, 0.1, 0.01) == 200 * 12000 * 10
    assert set_cost(10, 0.25, 0.1, 0.01) == 10 * 3 * 10


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out_path):
    import torch.distributed as dist
    from dense_b200 import workloads
    from dense_b200.sharding import gather_rows, shard
    from dense_b200.tissue import default_graph
    from oracle.pyoracle import load_oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    P = workloads.log_uniform_params(6, seed=41)
    durations = [2.0, 5.0, 1.0, 3.0, 4.0, 2.5]
    off, ids = default_graph(12, 4)
    costs = [12 * d for d in durations]
    mine = shard(costs, world)[rank]
    O = load_oracle("her_model_2014")
    rows = []
    for i in mine:
        sim = O.create(off, ids, np.tile(P[i], (12, 1)), P[i], None, 0.01)
        sim.run(durations[i], 0.1)
        rows.append(sim.state()[:, 0])
    full = gather_rows(rows, mine, 6)
    if rank == 0:
        np.save(out_path, full)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_shard_and_gather_match_one_process(tmp_path):
    out = str(tmp_path / "gathered.npy")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got = np.load(out)
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    from oracle.pyoracle import load_oracle
    P = workloads.log_uniform_params(6, seed=41)
    durations = [2.0, 5.0, 1.0, 3.0, 4.0, 2.5]
    off, ids = default_graph(12, 4)
    O = load_oracle("her_model_2014")
    for i in range(6):
        sim = O.create(off, ids, np.tile(P[i], (12, 1)), P[i], None, 0.01)
        sim.run(durations[i], 0.1)
        assert np.array_equal(got[i], sim.state()[:, 0])
