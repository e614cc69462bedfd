"""Parity of the CUDA engine (through its C ABI) with DENSE: bit for bit in
FP64 against DENSE's own outputs (fixtures) and the oracle; FP32+Kahan
within a stated tolerance; status words and drop semantics."""

import math

import numpy as np
import pytest

from dense_b200 import engine as E
from tests.golden.cases import build_case
from tests.helpers import load_fixture, mismatches, run_engine, run_oracle

pytestmark = pytest.mark.gpu

# her_pert_factors: -b perturbation factors resize DENSE's rings
# (base.cpp:55-140), moving the rows that zero-truncated delays read (lag S-1)
EXACT_CASES = ["her_test", "her_pert", "her_sets", "her_delays", "her_init", "her_pert_factors", "turing", "nan_test",
               "delay_reaction", "bz", "briggs_rauscher"]


@pytest.mark.parametrize("name", EXACT_CASES)
def test_fp64_bitwise_vs_dense_fixture(name):
    want = load_fixture(name)
    got = run_engine(name)
    for s in range(len(build_case(name)["sets"])):
        assert got["status_%d" % s] == 0
    assert mismatches(want, got) == []


@pytest.mark.parametrize("name", ["her_test", "her_pert", "her_sets", "her_delays", "her_cfg1_full", "bz",
                                  "delay_reaction"])
def test_shared_rows_and_register_kernels_both_match_dense(name):
    """Sets without in-order reads run in the register kernel, or on request
    in the wave kernel with their history rows in shared memory: both give
    DENSE's outputs bit for bit."""
    want = load_fixture(name)
    for schedule in (E.SCHEDULE_SHARED_ROWS, E.SCHEDULE_REGISTER):
        got = run_engine(name, schedule=schedule)
        assert mismatches(want, got) == [], schedule


@pytest.mark.parametrize("name", ["her_pert", "her_sets"])
def test_fp64_bitwise_vs_oracle(name):
    from oracle.pyoracle import load_oracle
    want = run_oracle(load_oracle("her_model_2014"), name)
    assert mismatches(want, run_engine(name)) == []


def test_graph_replay_and_chunked_runs_match_one_launch():
    full = run_engine("her_sets")
    assert mismatches(full, run_engine("her_sets", graph=True)) == []
    assert mismatches(full, run_engine("her_sets", chunks_per_call=37)) == []
    assert mismatches(full, run_engine("her_sets", graph=True, chunks_per_call=100)) == []


def _oracle_vs_engine(model, sets_spec, dt, interval, analyses, precision=0):
    """Runs the same sets through the engine (one batch) and the oracle (one
    simulation each); returns (engine results, oracle results) per set."""
    from oracle.pyoracle import load_oracle
    O = load_oracle(model)
    b = E.Batch(model, [s for s, _ in sets_spec], dt, interval, analyses, precision=precision)
    b.run()
    b.sync()
    out = []
    st = b.status()
    for i, (ps, cp) in enumerate(sets_spec):
        sim = O.create(ps.nbr_offsets, ps.nbr_ids, cp, ps.set_params, ps.init_conc, dt)
        for a in analyses:
            sp = O_species_ids(O, a.species)
            if a.kind == E.BASIC:
                sim.add_basic(sp, a.cell_start, a.cell_end, a.time_start, a.time_end)
            else:
                sim.add_oscillation(sp, a.cell_start, a.cell_end, a.time_start, a.time_end, a.win_range,
                                    a.anlys_intvl)
        sim.run(ps.duration, interval)
        eng = {"state": b.state(i), "status": st[i]}
        ora = {"state": sim.state()}
        for k, a in enumerate(analyses):
            if a.kind == E.BASIC:
                eng["b%d" % k], ora["b%d" % k] = b.basic(k, i), sim.basic(k)
            else:
                eng["o%d" % k], ora["o%d" % k] = b.oscillation(k, i), sim.oscillation(k)
        out.append((eng, ora))
    b.close()
    return out


def O_species_ids(O, names):
    return [O.species.index(x) if isinstance(x, str) else int(x) for x in names]


def _assert_same(pairs, analyses):
    from tests.helpers import same
    for eng, ora in pairs:
        assert eng["status"] == 0
        assert same(eng["state"], ora["state"])
        for k, a in enumerate(analyses):
            key = ("b%d" if a.kind == E.BASIC else "o%d") % k
            fields = ("mins", "sums", "maxs", "samples", "time") if a.kind == E.BASIC else \
                ("amps", "pers", "avg_peak", "ncrit", "samples", "time")
            for f in fields:
                assert same(eng[key][f], ora[key][f]), (key, f)


def test_memory_kernel_large_her_sets_bitwise():
    """Sets above one CTA of cells (300 and 1024) run in the memory-state
    kernel, mixed in one batch with a 200-cell set of the register kernel."""
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    rng = np.random.Generator(np.random.PCG64(31))
    base = workloads.template_params()
    spec = []
    for cells, width in ((200, 4), (300, 5), (1024, 8)):
        off, ids = default_graph(cells, width)
        cp = base[None, :] * rng.uniform(0.95, 1.05, size=(cells, base.size))
        spec.append((E.ParameterSet(off, ids, base, cell_params=cp, duration=6.0), cp))
    an = [E.Analysis.oscillation(["mh1", "ph1"], 0, 200, 0.0, float("inf"), 1.0, 0.1),
          E.Analysis.basic(["mh1", "pd", "md"], 0, 200)]
    _assert_same(_oracle_vs_engine("her_model_2014", spec, 0.01, 0.1, an), an)


@pytest.mark.parametrize("grid", [16, 40])
def test_turing_cell_ordered_reads_bitwise(grid):
    """Turing's neighbour averages read the row DENSE's cell loop is writing
    (lower-numbered neighbours already updated): the memory kernel's level
    schedule must reproduce that order exactly, also on grids past one CTA."""
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    p = workloads.template_params("turing")
    ic = np.array(workloads.templates()["turing"]["init_conc"])
    off, ids = default_graph(grid * grid, grid)
    spec = [(E.ParameterSet(off, ids, p, init_conc=ic, duration=3.0), np.tile(p, (grid * grid, 1)))]
    an = [E.Analysis.basic([0, 1, 2, 3], 0, grid * grid)]
    _assert_same(_oracle_vs_engine("turing", spec, 0.01, 0.1, an), an)


def test_fp32_kahan_error_vs_fp64():
    """FP32 rates with Kahan-compensated state: relative error of the final
    state and of the oscillation periods against FP64 (60 simulated minutes,
    200 perturbed cells)."""
    f64 = run_engine("her_pert", precision=E.FP64)
    f32 = run_engine("her_pert", precision=E.FP32_KAHAN)
    a, b = f64["state_0"], f32["state_0"]
    rel = np.max(np.abs(a - b) / np.maximum(np.abs(a), 1e-3))
    assert rel < 2e-3, rel
    per64, per32 = f64["a1_pers_0"], f32["a1_pers_0"]
    ok = np.isfinite(per64) & np.isfinite(per32)
    assert ok.sum() > 0
    assert np.max(np.abs(per64[ok] - per32[ok]) / per64[ok]) < 2e-2


def _her_batch(sets_params, cells=16, duration=30.0, analyses=()):
    from dense_b200.tissue import default_graph
    off, ids = default_graph(cells, 4)
    sets = [E.ParameterSet(off, ids, p, duration=duration) for p in sets_params]
    return E.Batch("her_model_2014", sets, 0.01, 0.1, list(analyses))


def test_nan_parameter_rejects_only_that_set():
    from dense_b200 import workloads
    p = workloads.template_params()
    bad = p.copy()
    bad[3] = float("nan")
    b = _her_batch([p, bad, p])
    b.run()
    b.sync()
    st = b.status()
    assert st[0] == 0 and st[2] == 0 and st[1] & E.SET_NAN_PARAM
    assert np.array_equal(b.state(0), b.state(2))
    ch, age = b.progress()
    assert ch[1] == 0 and ch[0] == 300


def test_concentration_check_drops_like_dense():
    """ConcentrationCheck (conccheck.hpp:25-51) with run_simulation's drop
    (run_simulation.hpp:131-150), against DENSE's own Deterministic_Simulation
    with that check (tests/golden/ref_her_conccheck.npz): four sets leave
    mh1's bounds in the first 15 minutes at different chunks, two leave the
    all-species bounds of cells 4-11 at minute 20, two run to the end; each
    dropped set stops at the chunk whose sample failed, with DENSE's state
    and Basic accumulators at that point."""
    want = load_fixture("her_conccheck")
    got = run_engine("her_conccheck")
    assert sorted(int(want["status_%d" % s]) for s in range(8)) == [0, 0, 1, 1, 1, 1, 1, 1]
    for s in range(8):
        assert (int(got["status_%d" % s]) & E.SET_DROPPED) == int(want["status_%d" % s])
        got["status_%d" % s] = np.int32(int(got["status_%d" % s]) & E.SET_DROPPED)
    assert mismatches(want, got) == []
    # a check whose bounds hold keeps every set
    from dense_b200 import workloads
    p = workloads.template_params()
    mh1 = workloads.her_species("mh1")[0]
    b2 = _her_batch([p], analyses=[E.Analysis.conccheck([mh1], 0, 16, 0.0, 1e9)])
    b2.run()
    assert b2.status()[0] == 0


def test_uneven_horizons_in_one_batch():
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    from oracle.pyoracle import load_oracle
    O = load_oracle("her_model_2014")
    P = workloads.log_uniform_params(3, seed=9)
    off, ids = default_graph(12, 4)
    durs = [5.0, 12.3, 0.0]
    sets = [E.ParameterSet(off, ids, P[i], duration=durs[i]) for i in range(3)]
    b = E.Batch("her_model_2014", sets, 0.01, 0.1)
    b.run()
    ch, age = b.progress()
    for i in range(3):
        sim = O.create(off, ids, np.tile(P[i], (12, 1)), P[i], None, 0.01)
        n = sim.run(durs[i], 0.1)
        assert ch[i] == n == math.ceil(durs[i] / 0.1)
        assert age[i] == sim.age()
        assert np.array_equal(b.state(i), sim.state())


@pytest.mark.parametrize("model", ["delay_reaction", "bz", "briggs_rauscher", "nan_test", "turing"])
def test_other_models_bitwise_vs_oracle(model):
    """DENSE's other example models, compiled unchanged through the model
    headers, against the oracle: random positive parameters, 24 cells,
    initial concentrations in [0, 5)."""
    from dense_b200.tissue import default_graph
    L = E.load(model)
    rng = np.random.Generator(np.random.PCG64(sum(model.encode())))
    p = rng.uniform(0.05, 2.0, size=L.num_params)
    if L.num_delay_reactions:
        p[L.num_reactions:L.num_reactions + L.num_delay_reactions] = rng.uniform(0.5, 4.0, L.num_delay_reactions)
    off, ids = default_graph(24, 6)
    ic = rng.uniform(0.0, 5.0, size=L.num_species)
    spec = [(E.ParameterSet(off, ids, p, init_conc=ic, duration=4.0), np.tile(p, (24, 1)))]
    an = [E.Analysis.basic(list(range(L.num_species)), 0, 24)]
    _assert_same(_oracle_vs_engine(model, spec, 0.01, 0.1, an), an)


@pytest.mark.parametrize("cells,width", [(1, 1), (2, 1), (5, 4), (3, 3)])
def test_tiny_and_ragged_tissues_bitwise(cells, width):
    """Tissues of one to five cells, widths that do not divide the cell
    count: same states and analyses as the oracle."""
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    p = workloads.log_uniform_params(1, seed=cells)[0]
    off, ids = default_graph(cells, width)
    spec = [(E.ParameterSet(off, ids, p, duration=6.0), np.tile(p, (cells, 1)))]
    an = [E.Analysis.basic(["mh1", "pd"], 0, cells),
          E.Analysis.oscillation(["mh1"], 0, cells, 0.0, float("inf"), 1.0, 0.1)]
    _assert_same(_oracle_vs_engine("her_model_2014", spec, 0.01, 0.1, an), an)


def test_cells_without_neighbours_bitwise():
    """Cells with an empty neighbour list (DENSE averages 0 / 0 = NaN and
    reads 0) next to connected ones."""
    from dense_b200 import workloads
    p = workloads.log_uniform_params(1, seed=21)[0]
    nbrs = [[], [2], [1, 3], [], [0, 1, 2, 3, 5], [4]]
    off = np.cumsum([0] + [len(x) for x in nbrs]).astype(np.int32)
    ids = np.array([v for x in nbrs for v in x], np.int32)
    spec = [(E.ParameterSet(off, ids, p, duration=6.0), np.tile(p, (6, 1)))]
    an = [E.Analysis.basic(["pd", "mh1"], 0, 6)]
    _assert_same(_oracle_vs_engine("her_model_2014", spec, 0.01, 0.1, an), an)


def test_fp32_kahan_turing_close_to_fp64():
    """FP32 with Kahan-compensated state in the wave kernel (in-order
    neighbour reads), against FP64: 16 x 16 and 48 x 48 grids, 3 minutes."""
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    p = workloads.template_params("turing")
    ic = np.array(workloads.templates()["turing"]["init_conc"])
    sets = []
    for N in (16, 48):
        off, ids = default_graph(N * N, N)
        sets.append(E.ParameterSet(off, ids, p, init_conc=ic, duration=3.0))
    res, basic = {}, {}
    for prec in (E.FP64, E.FP32_KAHAN):
        # Basic over 0..255 of every set: the analyses sample the
        # compensated values (the Kahan terms live in shared memory)
        an = [E.Analysis.basic(list(range(4)), 0, 256)]
        b = E.Batch("turing", sets, 0.01, 0.1, an, precision=prec)
        b.run()
        b.sync()
        assert (b.status() == 0).all()
        res[prec] = [b.state(i) for i in range(len(sets))]
        basic[prec] = [np.concatenate([b.basic(0, i)[k].ravel() for k in ("cell_mins", "cell_maxs", "cell_sums")])
                       for i in range(len(sets))]
        b.close()
    for a, f in zip(res[E.FP64] + basic[E.FP64], res[E.FP32_KAHAN] + basic[E.FP32_KAHAN]):
        rel = np.max(np.abs(a - f) / np.maximum(np.abs(a), 1e-3))
        assert rel < 1e-4, rel


def test_checkpoint_and_resume_continue_bit_for_bit():
    """A checkpoint taken mid-run and restored -- into a new batch built from
    the same inputs, or into the same batch after it ran on -- continues to
    the same final state and analysis outputs as the uninterrupted run; a
    snapshot of another layout or a truncated one is refused."""
    full = run_engine("her_sets")
    from tests.golden.cases import build_case
    case = build_case("her_sets")

    def batch():
        sets = [E.ParameterSet(ps["off"], ps["ids"], ps["set_params"], duration=ps["duration"])
                for ps in case["sets"]]
        an = [E.Analysis.basic(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1])
              if a["kind"] == "basic" else
              E.Analysis.oscillation(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"],
                                     a["intvl"]) for a in case["analyses"]]
        return E.Batch(case["model"], sets, case["dt"], case["interval"], an)

    a = batch()
    a.run(517)
    snap = a.checkpoint()
    a.run(-1)
    b = batch()
    b.restore(snap)
    b.run(-1)
    a.restore(snap)   # back in time on the same engine
    a.run(-1)
    for x in (a, b):
        for s in range(len(case["sets"])):
            assert np.array_equal(x.state(s), full["state_%d" % s])
            o = x.oscillation(1, s)
            assert np.array_equal(o["pers"], full["a1_pers_%d" % s], equal_nan=True)
            assert np.array_equal(o["amps"], full["a1_amps_%d" % s], equal_nan=True)
            r = x.basic(0, s)
            assert np.array_equal(r["sums"], full["a0_sums_%d" % s])
    with pytest.raises(E.DenseError):
        b.restore(snap[:100])
    from dense_b200 import workloads
    other = _her_batch([workloads.template_params()])
    with pytest.raises(E.DenseError):
        other.restore(snap)
    for x in (a, b, other):
        x.close()
