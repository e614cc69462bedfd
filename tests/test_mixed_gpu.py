"""Uneven mixed batches: schedule hints, the autotuner and the one-graph
her_model_2014 + Turing-Pattern batch give the same results as the oracle
and as plain per-model runs."""

import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

from dense_b200 import engine as E
from dense_b200 import workloads
from dense_b200.tissue import default_graph
from tests.test_engine_gpu import _assert_same, _oracle_vs_engine


def _her_set(cells, width, rng, duration):
    p = workloads.template_params() * np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=45))
    L = E.load("her_model_2014")
    p[L.num_reactions:L.num_reactions + L.num_delay_reactions] = rng.uniform(
        5.0, 20.0, size=L.num_delay_reactions)
    off, ids = default_graph(cells, width)
    return E.ParameterSet(off, ids, p, duration=duration), np.tile(p, (cells, 1))


@pytest.mark.parametrize("cells,width,hints", [
    (40, 4, [(0, 0), (1, 32), (1, 64)]),
    (300, 5, [(0, 0), (1, 64), (1, 128), (1, 256)]),
])
def test_her_every_schedule_bitwise(cells, width, hints):
    """The same her set under the register kernel and memory-kernel CTAs
    of several widths (cells per thread 1..10), delays U[5, 20] min."""
    rng = np.random.Generator(np.random.PCG64(cells))
    ps, cp = _her_set(cells, width, rng, 8.0)
    spec = []
    for sched, blk in hints:
        q = copy.copy(ps)
        q.schedule, q.mem_block = sched, blk
        spec.append((q, cp))
    an = [E.Analysis.oscillation(["mh1", "ph1"], 0, 40, 0.0, float("inf"), 1.0, 0.1),
          E.Analysis.basic(["mh1", "pd", "md"], 0, 40)]
    _assert_same(_oracle_vs_engine("her_model_2014", spec, 0.01, 0.1, an), an)


TURING_HINTS = [(0, 0), (1, 32), (1, 64), (E.SCHEDULE_GLOBAL, 0), (E.SCHEDULE_SHARED_NEIGHBOUR, 0),
                (E.SCHEDULE_GLOBAL, 64), (E.SCHEDULE_WAVE_GLOBAL, 32), (E.SCHEDULE_WAVE_GLOBAL, 64)]


@pytest.mark.parametrize("grid,minutes", [(12, 3.0), (37, 3.0), (64, 0.5)])
def test_turing_every_schedule_bitwise(grid, minutes):
    """Turing's ordered neighbour reads in the wave kernel (rows in shared
    memory as far as they fit: all species at 12 x 12, the in-order species
    and records at 37 x 37, only the in-order species at 64 x 64), with
    only neighbour-read species shared, with every row global (single-warp
    CTAs at 64 registers, or two warps), and in the memory kernel with every
    row global; CTAs of one and two warps."""
    p = workloads.template_params("turing")
    ic = np.array(workloads.templates()["turing"]["init_conc"])
    off, ids = default_graph(grid * grid, grid)
    spec = []
    for sched, b in TURING_HINTS:
        spec.append((E.ParameterSet(off, ids, p, init_conc=ic, duration=minutes, schedule=sched, mem_block=b),
                     np.tile(p, (grid * grid, 1))))
    an = [E.Analysis.basic([0, 1, 2, 3], 0, 144), E.Analysis.oscillation([1], 0, 144, 0.0, float("inf"), 0.2, 0.1)]
    _assert_same(_oracle_vs_engine("turing", spec, 0.01, 0.1, an), an)


def _small_mixed(num_sets, seed):
    """A mixed batch of the full generator with horizons cut to 2..6 min."""
    groups = workloads.mixed_sets(num_sets, seed=seed)
    rng = np.random.Generator(np.random.PCG64(seed))
    for sets in groups.values():
        for s in sets:
            s.duration = float(rng.uniform(2.0, 6.0))
    return groups


def test_mixed_graph_matches_plain_runs_and_autotune():
    """One captured graph over both models' engines, replayed in chunks,
    with autotuned schedules, ends in the same states as each model's plain
    one-launch run with default schedules."""
    from dense_b200.autotune import Autotuner
    from dense_b200.mixed import MixedBatch
    groups = _small_mixed(48, seed=5)
    assert groups["her_model_2014"] and groups["turing"]
    plain = {}
    for m, sets in groups.items():
        b = E.Batch(m, sets, 0.01, 0.1)
        b.run(-1)
        b.sync()
        assert (b.status() == 0).all()
        plain[m] = [b.state(i) for i in range(len(sets))]
        b.close()
    tuned = {m: [copy.copy(s) for s in sets] for m, sets in groups.items()}
    tuner = Autotuner(sample_sets=2, minutes=0.2)
    for m, sets in tuned.items():
        chosen = tuner.tune(m, sets, 0.01)
        assert chosen and all(s.schedule in (0, 1, 2, 3, 4) for s in sets)
    mb = MixedBatch(tuned, 0.01, 0.1)
    for _ in range(7):  # 7 x 9 chunks cover the 6-minute horizons
        mb.run(9)
    mb.sync()
    for m, b in mb.batches.items():
        assert (b.status() == 0).all()
        for i in range(len(b.sets)):
            assert np.array_equal(b.state(i), plain[m][i], equal_nan=True), (m, i)
    assert mb.done_cell_steps(10) == mb.info()["total_cell_steps"]
    mb.close()
