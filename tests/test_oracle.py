"""The oracle, pinned: against DENSE's CTest golden files and against
full-precision outputs of DENSE itself (fixtures, and the live harness when
it is built here)."""

import os

import numpy as np
import pytest

from dense_b200 import report
from tests.golden.cases import CASES, build_case
from tests.helpers import GOLDEN, load_fixture, mismatches, run_oracle

pytestmark = pytest.mark.filterwarnings("ignore::RuntimeWarning")


@pytest.fixture(scope="module")
def her():
    from oracle.pyoracle import load_oracle
    return load_oracle("her_model_2014")


def _lib(model):
    from oracle.pyoracle import load_oracle
    return load_oracle(model)


def _ctest(name):
    with open(os.path.join(GOLDEN, "dense_ctest", name)) as f:
        return f.read()


def _her_ctest_run(her, cells, width, minutes):
    """DENSE's her CTest arguments: -c cells -w width -t minutes -u .01 -s .01
    with test/her_model_2014/analyses.xml (the Basic of cells 0-9 over 0-15
    minutes and the Oscillation of cells 0-5 over 0-60 minutes)."""
    p = np.array(__import__("dense_b200.workloads", fromlist=["x"]).template_params())
    off, ids = her.default_graph(cells, width)
    sim = her.create(off, ids, np.tile(p, (cells, 1)), p, None, 0.01)
    sp = {n: i for i, n in enumerate(her.species)}
    sim.add_basic([sp["ph1"], sp["ph7"]], 0, 9, 0.0, 15.0)
    sim.add_oscillation([sp["ph1"], sp["mh1"], sp["md"]], 0, 5, 0.0, 60.0, 4.0, 0.01)
    sim.run(minutes, 0.01)
    return sim, [sp["ph1"], sp["ph7"]], [sp["ph1"], sp["mh1"], sp["md"]]


def test_her_test_golden_csv_bytes(her):
    sim, bsp, osp = _her_ctest_run(her, 10, 5, 3000.0)
    b = report.basic_csv(her.species, bsp, sim.basic(0), 0, 9)
    o = report.oscillation_csv(her.species, osp, sim.oscillation(1), 0, 5)
    assert b == _ctest("her_anlys_basic_a.csv")
    assert o == _ctest("her_anlys_oscil.csv")


@pytest.mark.parametrize("cells,width,minutes,golden", [
    (10, 1, 3000.0, "her_anlys_basic_a.csv"),           # cell_width_test
    (50, 10, 3000.0, "her_cell_width_test_anlys.csv"),  # cell_width_test_01
    (10, 5, 300.0, "her_total_time_test_anlys.csv"),    # time_total_test
])
def test_her_ctest_variants(her, cells, width, minutes, golden):
    sim, bsp, _ = _her_ctest_run(her, cells, width, minutes)
    assert report.basic_csv(her.species, bsp, sim.basic(0), 0, 9) == _ctest(golden)


def test_nan_golden_csv():
    L = _lib("nan_test")
    case = build_case("nan_test")
    ps = case["sets"][0]
    sim = L.create(ps["off"], ps["ids"], ps["cell_params"], ps["set_params"], None, 0.01)
    sim.add_basic([0, 1, 2], 0, 99, 0.0, 2.0)
    sim.run(15.0, 0.5)
    text = report.basic_csv(L.species, [0, 1, 2], sim.basic(0), 0, 99)
    # DENSE's NaNs come out of x86 arithmetic with the sign bit set ("-nan");
    # NaN payloads are not part of the comparison.
    assert text.replace("-nan", "nan") == _ctest("nan_anlys_basic_a.csv").replace("-nan", "nan")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_dense_fixture(name):
    want = load_fixture(name)
    got = run_oracle(_lib(build_case(name)["model"]), name)
    assert mismatches(want, got) == []


def test_oracle_matches_live_dense():
    """A fresh random case against DENSE itself, where its build exists."""
    from oracle.pyoracle import load_ref
    R = load_ref("her_model_2014")
    if R is None:
        pytest.skip("DENSE harness not built on this machine")
    O = _lib("her_model_2014")
    rng = np.random.Generator(np.random.PCG64(11))
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    p = workloads.template_params() * np.exp(rng.uniform(np.log(0.5), np.log(2.0), 45))
    cp = p[None, :] * rng.uniform(0.9, 1.1, size=(24, 45))
    off, ids = default_graph(24, 6)
    ic = rng.uniform(0, 50, 14)
    res = []
    for L in (O, R):
        sim = L.create(off, ids, cp, p, ic, 0.02)
        sim.add_oscillation([4, 0, 7], 0, 24, 1.0, 50.0, 3.0, 0.2)
        sim.add_basic(list(range(14)), 0, 24, 0.0, 80.0)
        sim.run(90.0, 0.2)
        res.append((sim.state(), sim.oscillation(0), sim.basic(1), sim.ring_sizes()[0]))
    assert np.array_equal(res[0][0], res[1][0])
    assert np.array_equal(res[0][3], res[1][3])
    for k in ("amps", "pers", "avg_peak", "ncrit"):
        assert np.array_equal(res[0][1][k], res[1][1][k], equal_nan=True), k
    for k in ("mins", "sums", "maxs", "cell_mins", "cell_sums", "cell_maxs"):
        assert np.array_equal(res[0][2][k], res[1][2][k]), k


def test_default_graph_matches_oracle(her):
    from dense_b200.tissue import default_graph
    for cells, width in [(10, 5), (10, 1), (200, 4), (64, 8), (7, 3), (1, 1)]:
        a = default_graph(cells, width)
        b = her.default_graph(cells, width)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (cells, width)


def test_default_graph_known_answer():
    # cell 0 of the 200-cell, width-4 tissue reaches {3, 196, 197, 199};
    # half the cells have 4 out-neighbours and half have 5
    from dense_b200.tissue import default_graph
    off, ids = default_graph(200, 4)
    assert list(ids[off[0]:off[1]]) == [3, 196, 197, 199]
    deg = np.diff(off)
    assert (deg == 4).sum() == 100 and (deg == 5).sum() == 100


def test_ring_sizes_known_answer(her):
    # baby_cl sizes for the template parameters at dt = 0.01
    from dense_b200 import workloads
    p = workloads.template_params()
    off, ids = her.default_graph(10, 5)
    sim = her.create(off, ids, np.tile(p, (10, 1)), p, None, 0.01)
    S, _ = sim.ring_sizes()
    want = dict(ph1=2, ph7=2, ph13=2, ph17=2, ph113=2, ph77=2, ph1313=2, pd=1066, mh1=174, mh7=195, mh13=82,
                md=1138, ph11=1127, ph713=1127)
    assert {n: int(S[i]) for i, n in enumerate(her.species)} == want


def _random_tissue(rng, n, max_deg):
    """Ascending, duplicate-free out-neighbour lists of 0..max_deg cells each
    (self-loops allowed, as in a graph file)."""
    off, ids = [0], []
    for _ in range(n):
        k = int(rng.integers(0, max_deg + 1))
        ids.extend(sorted(rng.choice(n, size=min(k, n), replace=False).tolist()))
        off.append(len(ids))
    return np.array(off, np.int32), np.array(ids, np.int32)


@pytest.mark.parametrize("model,seed", [("her_model_2014", 31), ("turing", 32)])
def test_oracle_matches_live_dense_on_irregular_tissues(model, seed):
    """Random tissues with 0-12 out-neighbours per cell (graph-file inputs),
    against DENSE itself: her's delayed neighbour averages, and Turing's
    in-order reads of the row being written, where the order of a cell's
    neighbours relative to it decides old or new values."""
    from oracle.pyoracle import load_ref
    R = load_ref(model)
    if R is None:
        pytest.skip("DENSE harness not built on this machine")
    O = _lib(model)
    from dense_b200 import workloads
    rng = np.random.Generator(np.random.PCG64(seed))
    n = 30
    off, ids = _random_tissue(rng, n, 12)
    p = workloads.template_params(model)
    if model == "turing":
        p = p * np.exp(rng.uniform(np.log(0.5), np.log(2.0), p.size))
        ic = np.array(workloads.templates()["turing"]["init_conc"], np.float64) + rng.uniform(0, 1, 4)
    else:
        p = p * np.exp(rng.uniform(np.log(0.5), np.log(2.0), p.size))
        ic = rng.uniform(0, 20, 14)
    cp = p[None, :] * rng.uniform(0.9, 1.1, size=(n, p.size))
    res = []
    for L in (O, R):
        sim = L.create(off, ids, cp, p, ic, 0.01)
        nsp = L.num_species
        sim.add_basic(list(range(nsp)), 0, n, 0.0, float("inf"))
        sim.run(20.0, 0.1)
        res.append((sim.state(), sim.basic(0)))
    assert np.array_equal(res[0][0], res[1][0], equal_nan=True)
    for k in ("mins", "sums", "maxs", "cell_mins", "cell_sums", "cell_maxs"):
        assert np.array_equal(res[0][1][k], res[1][1][k], equal_nan=True), k
