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


def _oracle_runner(model, sets, step_size, interval, analyses, precision, device, with_state):
    """Stands in for the engine runner on CPU ranks (same keys)."""
    from oracle.pyoracle import load_oracle
    O = load_oracle(model)
    out = {"status": [], "amps_0": [], "pers_0": [], "state": []}
    for s in sets:
        cp = s.cell_params if s.cell_params is not None else np.tile(s.set_params, (s.num_cells, 1))
        sim = O.create(s.nbr_offsets, s.nbr_ids, cp, s.set_params, s.init_conc, step_size)
        a = analyses[0]
        sim.add_oscillation([1, 4], a.cell_start, a.cell_end, a.time_start, a.time_end, a.win_range, a.anlys_intvl)
        sim.run(s.duration, interval)
        o = sim.oscillation(0)
        out["status"].append(sim.status())
        out["amps_0"].append(o["amps"])
        out["pers_0"].append(o["pers"])
        out["state"].append(sim.state())
    out["status"] = np.asarray(out["status"], np.int32)
    return out


def _sharded_inputs():
    from dense_b200 import engine as E, workloads
    from dense_b200.tissue import default_graph
    P = workloads.log_uniform_params(7, seed=43)
    sets = []
    for i, (cells, dur) in enumerate([(12, 6.0), (16, 2.0), (8, 9.0), (12, 1.0), (20, 4.0), (8, 3.0), (16, 5.0)]):
        off, ids = default_graph(cells, 4)
        sets.append(E.ParameterSet(off, ids, P[i], duration=dur))
    an = [E.Analysis.oscillation([1, 4], 0, 8, 0.0, float("inf"), 1.0, 0.1)]
    return sets, an


def _sharded_rank(rank, world, port, out_path):
    import pickle
    import torch.distributed as dist
    from dense_b200.sharding import simulate_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sets, an = _sharded_inputs()
    res = simulate_sharded("her_model_2014", sets, 0.01, 0.1, an, with_state=True, run_batch=_oracle_runner)
    with open(out_path % rank, "wb") as f:
        pickle.dump(res, f)
    dist.barrier()
    dist.destroy_process_group()


def test_simulate_sharded_two_ranks_equal_one_process(tmp_path):
    """simulate_sharded over two gloo ranks (cost-balanced shares, one gather
    at the end) returns, on every rank, what one process returns."""
    import pickle
    from dense_b200.sharding import simulate_sharded
    out = str(tmp_path / "rank%d.pkl")
    mp.start_processes(_sharded_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    sets, an = _sharded_inputs()
    one = simulate_sharded("her_model_2014", sets, 0.01, 0.1, an, with_state=True, run_batch=_oracle_runner)
    assert one["shares"] == [list(range(7))]
    for r in range(2):
        with open(out % r, "rb") as f:
            got = pickle.load(f)
        assert sorted(got["shares"][0] + got["shares"][1]) == list(range(7)) and all(got["shares"])
        assert np.array_equal(got["status"], one["status"])
        for k in ("amps_0", "pers_0"):
            assert np.array_equal(got[k], one[k], equal_nan=True), k
        for a, b in zip(got["state"], one["state"]):
            assert np.array_equal(a, b)
