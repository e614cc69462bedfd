"""FP64 engine parity with DENSE at the configurations' full sizes, against
fixtures DENSE itself made (tests/golden/make_goldens.py, FULL_CASES in
tests/golden/cases.py):

* the one-set configuration: 200 cells with every parameter of every cell
  x U(0.95, 1.05), the whole 600 minutes, Basic over every species and
  cell + Oscillation of mh1 and ph1 every 0.1 min;
* eight of the batched configuration's own 4096 sets (those with the
  fewest and the most minutes of truncated delay), 200 cells, the whole
  1200 minutes, Oscillation of mh1 every 0.1 min -- run inside a batch of
  more sets than one wave of CTAs holds, in graph-replayed launches of 100
  minutes as the benchmark runs them, so the history rings live in L2
  under the benchmark's own pressure;
* the uneven mixed batch's largest shapes at 1200 minutes: a her_model_2014
  set of 1024 cells with every delay in [5, 20] min (the memory kernel),
  once with one parameter row (every cell then follows the same
  trajectory) and once with every parameter of every cell x U(0.95, 1.05),
  and a 64 x 64 Turing-Pattern grid (the wave kernel).

Semantics pinned: run_simulation.hpp:127-157 (chunks, analyses before each
age_by), oscillation.ipp:7-185 (windows over 12,000 samples), the lag reads
of determ.hpp:73-89 over the whole horizon."""

import numpy as np
import pytest

from dense_b200 import engine as E, workloads
from tests.golden.cases import CFG2_SETS, build_case
from tests.helpers import load_fixture, mismatches, run_engine

pytestmark = pytest.mark.gpu


def _check_all_sets(name):
    want = load_fixture(name)
    got = run_engine(name)
    for s in range(len(build_case(name)["sets"])):
        assert got["status_%d" % s] == 0
    assert mismatches(want, got) == []


def test_one_set_configuration_600_minutes():
    _check_all_sets("her_cfg1_full")


def test_batched_configuration_sets_1200_minutes_inside_a_full_wave():
    want = load_fixture("her_cfg2_full")
    idx = [int(i) for i in want["indices"]]
    # the benchmark's first 296 sets (two CTAs on each of 148 SMs) plus the
    # fixture's sets, all at the full horizon
    members = sorted(set(range(296)) | set(idx))
    every = workloads.log_uniform_sets(CFG2_SETS, cells=200, width=4, duration=1200.0, seed=2)
    sets = [every[i] for i in members]
    b = E.Batch("her_model_2014", sets, 0.01, 0.1, workloads.batch_analyses(200, 0.1))
    for _ in range(12):
        b.run(1000, graph=True)
    b.sync()
    status = b.status()
    chunks, _ = b.progress()
    got = {}
    for s, i in enumerate(idx):
        k = members.index(i)
        assert status[k] == 0
        got["chunks_%d" % s] = chunks[k]
        got["state_%d" % s] = b.state(k)
        got["S_%d" % s] = b.ring_info(k)[0]
        o = b.oscillation(0, k)
        for key in ("amps", "pers", "avg_peak", "ncrit", "samples", "time"):
            got["a0_%s_%d" % (key, s)] = np.asarray(o[key])
    b.close()
    want.pop("indices")
    assert mismatches(want, got) == []


def test_mixed_batch_largest_her_set_1024_cells_1200_minutes():
    _check_all_sets("her_cfg3_large")


def test_mixed_batch_largest_her_set_with_per_cell_parameters():
    _check_all_sets("her_cfg3_large_cells")


def test_mixed_batch_largest_turing_grid_64x64_1200_minutes():
    _check_all_sets("turing_cfg3_large")
