"""Error behaviour of the C ABI on malformed input, through
dense_engine_plan (the same validation dense_engine_create runs before it
touches a GPU): every bad descriptor is refused with its DENSE_ERR_* code
and a message, nothing is undefined behaviour."""

import numpy as np
import pytest

from dense_b200 import engine as E, workloads
from dense_b200.tissue import default_graph

INVALID, UNSUPPORTED = 1, 4


def _set(cells=8, width=4, **kw):
    off, ids = default_graph(cells, width)
    kw.setdefault("duration", 10.0)
    return E.ParameterSet(off, ids, workloads.template_params(), **kw)


def _code(sets, analyses=(), dt=0.01, interval=0.1, precision=E.FP64):
    try:
        E.plan("her_model_2014", sets, dt, interval, analyses, precision)
    except E.DenseError as e:
        text = str(e)
        return int(text.split("error ")[1].split(":")[0]), text
    return 0, ""


def _csr(offsets, ids, **kw):
    return E.ParameterSet(np.array(offsets), np.array(ids), workloads.template_params(), duration=10.0, **kw)


def test_a_valid_batch_plans():
    assert _code([_set(), _set(200, 4)]) == (0, "")


@pytest.mark.parametrize("offsets,ids,msg", [
    ([0, 1, 2], [1, 5], "neighbour id outside the tissue"),
    ([0, 1, 2], [1, -1], "neighbour id outside the tissue"),
    ([0, 2, 2], [1, 1], "must ascend"),
    ([0, 2, 1], [0, 1], "CSR offsets decrease"),
    ([1, 2, 3], [1, 0, 0], "CSR offsets must start at 0"),
])
def test_bad_neighbour_lists(offsets, ids, msg):
    code, text = _code([_csr(offsets, ids)])
    assert code == INVALID and msg in text


def test_cell_count_limits():
    code, text = _code([_csr([0], [])])
    assert code == UNSUPPORTED and "cells per set" in text


@pytest.mark.parametrize("duration", [-1.0, float("nan")])
def test_bad_duration(duration):
    code, text = _code([_set(duration=duration)])
    assert code == INVALID and "duration" in text


@pytest.mark.parametrize("duration", [-1.0, float("nan"), 1e300])
def test_bad_duration_with_a_trajectory(duration):
    """The trajectory capacity is sized from the sets' horizons before the
    sets are checked; an invalid or absurd horizon is an error code."""
    an = [E.Analysis.trajectory(["mh1"], 0, 8)]
    code, _ = _code([_set(), _set(duration=duration)], an)
    assert code in (INVALID, UNSUPPORTED)


@pytest.mark.parametrize("dt,interval", [(0.0, 0.1), (-0.01, 0.1), (0.01, 0.0), (float("nan"), 0.1)])
def test_bad_step_or_interval(dt, interval):
    code, text = _code([_set()], dt=dt, interval=interval)
    assert code == INVALID and "positive" in text


def test_unknown_precision():
    code, text = _code([_set()], precision=7)
    assert code == INVALID and "precision" in text


@pytest.mark.parametrize("schedule,mem_block,msg", [
    (7, 0, "schedule hint"), (-1, 0, "schedule hint"), (1, 48, "mem_block"), (1, 512, "mem_block"),
    (1, 16, "mem_block"),
])
def test_bad_schedule_hints(schedule, mem_block, msg):
    code, text = _code([_set(schedule=schedule, mem_block=mem_block)])
    assert code == INVALID and msg in text


def test_analysis_checks():
    s = [_set(8, 4)]
    assert _code(s, [E.Analysis.basic(["mh1"], 0, 9)])[0] == INVALID          # past the tissue
    assert _code(s, [E.Analysis.basic(["mh1"], 5, 4)])[0] == INVALID          # end before start
    assert _code(s, [E.Analysis.basic([14], 0, 8)])[0] == INVALID             # species id
    assert _code(s, [E.Analysis.basic([], 0, 8)])[0] == INVALID               # no species
    assert _code(s, [E.Analysis.oscillation(["mh1"], 0, 8, 0, 10, 4.0, 0.0)])[0] == INVALID
    assert _code(s, [E.Analysis.oscillation(["mh1"], 0, 8, 0, 10, 1e9, 1e-3)])[0] == UNSUPPORTED
    assert _code(s, [E.Analysis.basic(["mh1"], 0, 8)] * 9)[0] == UNSUPPORTED   # more than 8 analyses
    assert _code(s, [E.Analysis.conccheck([], 0, 8, 0.0, 1e3)])[0] == 0     # all species


def test_analysis_range_is_checked_against_the_smallest_set():
    code, text = _code([_set(200, 4), _set(8, 4)], [E.Analysis.basic(["mh1"], 0, 100)])
    assert code == INVALID and "outside the tissue" in text


# dense_simulate_noalloc checks its batch on the host before it touches a
# device, so its refusals need no GPU either.
SCRATCH_TOO_SMALL = 5


def _noalloc_code(sets, precision=E.FP64, analyses=(), model="her_model_2014"):
    import ctypes as C
    L = E.load(model)
    run, cset, keep = E._describe(L, sets, list(analyses), 0.01, 0.1, precision, 0)
    f = L.lib.dense_simulate_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(E._RunDesc), C.c_int, C.POINTER(E._SetDesc), C.POINTER(C.c_double),
                  C.POINTER(C.c_int32), C.c_void_p]
    out = np.zeros(max(1, sum(L.num_species * s.num_cells for s in sets)))
    return f(C.byref(run), len(sets), cset, out.ctypes.data_as(C.POINTER(C.c_double)), None, None)


def test_noalloc_refusals_on_the_host():
    assert _noalloc_code([_set()] * 65) == SCRATCH_TOO_SMALL                 # more than 64 sets
    assert _noalloc_code([_set()], precision=E.FP32_KAHAN) == UNSUPPORTED
    assert _noalloc_code([_set()], analyses=[E.Analysis.basic(["mh1"], 0, 8)]) == UNSUPPORTED
    assert _noalloc_code([_set(260, 4)]) == INVALID                          # more than 256 cells
    assert _noalloc_code([_set(duration=-1.0)]) == INVALID
    assert _noalloc_code([_csr([0, 1, 2], [1, 5])]) == INVALID               # id outside the tissue
    assert _noalloc_code([_csr([0, 2, 1], [0, 1])]) == INVALID               # offsets decrease
    assert _noalloc_code([_csr([0, 2, 2], [1, 1])]) == INVALID               # ids not ascending
    assert _noalloc_code([_set(256, 4, duration=1.0)] * 64) == SCRATCH_TOO_SMALL  # past 16 MiB


def test_noalloc_refuses_in_order_neighbour_reads_on_the_host():
    """A Turing-Pattern set reads its neighbours' rows of the same step
    (DENSE's in-order cell loop): the register kernel, the only kernel the
    no-allocation entry point runs, cannot run it, so the call is refused
    instead of returning an unsimulated state."""
    off, ids = default_graph(16, 4)
    p = workloads.template_params("turing")
    ic = np.array(workloads.templates()["turing"]["init_conc"])
    ordered = E.ParameterSet(off, ids, p, init_conc=ic, duration=1.0)
    assert _noalloc_code([ordered], model="turing") == UNSUPPORTED
    # and so is a batch where only one of several sets is ordered
    assert _noalloc_code([ordered] * 3, model="turing") == UNSUPPORTED


def test_every_entry_point_refuses_null_arguments():
    """NULL engines, graphs and output pointers give DENSE_ERR_INVALID (and
    destroying NULL is a no-op), before any device call."""
    lib = E.load("her_model_2014").lib
    calls = {
        "dense_engine_run": (None, 1, None), "dense_engine_run_graph": (None, 1, None),
        "dense_engine_sync": (None,), "dense_engine_reset": (None, None), "dense_engine_status": (None, None),
        "dense_engine_progress": (None, None, None), "dense_engine_read_state": (None, 0, None),
        "dense_engine_read_basic": (None, 0, 0, None, None, None, None, None, None, None, None),
        "dense_engine_read_oscillation": (None, 0, 0, None, None, None, None, None, None),
        "dense_engine_read_trajectory": (None, 0, 0, None, None, 0, None),
        "dense_engine_read_oscillation_all": (None, 0, None, None),
        "dense_engine_copy_trajectory": (None, 0, None, 0, None, None),
        "dense_engine_trajectory_capacity": (None, 0, None), "dense_engine_info": (None, None, None, None),
        "dense_engine_ring_info": (None, 0, None, None), "dense_graph_launch": (None, None),
        "dense_engine_checkpoint_size": (None, None), "dense_engine_checkpoint": (None, None, 0),
        "dense_engine_restore": (None, None, 0),
        "dense_graph_capture": (0, None, None, 0, 0, None), "dense_engine_create": (None, 0, None, None),
        "dense_engine_plan": (None, 0, None, None, None, None), "dense_model_get_info": (None,),
    }
    for name, args in calls.items():
        assert getattr(lib, name)(*args) == INVALID, name
        assert lib.dense_last_error(), name
    assert lib.dense_engine_destroy(None) == 0
    assert lib.dense_graph_destroy(None) == 0
    assert lib.dense_model_specie_name(-1) is None and lib.dense_model_reaction_name(10 ** 6) is None


def test_largest_set_plans_and_one_more_cell_is_refused():
    """65536 cells is the largest set (16-bit cell ids in the wave kernel's
    records, and the memory kernel's limit): it plans, in the memory-state
    kernel; 65537 cells is refused as unsupported."""
    for model in ("her_model_2014", "turing"):
        p = workloads.template_params(model)
        off, ids = default_graph(65536, 256)
        nbytes, kernel, levels = E.plan(model, [E.ParameterSet(off, ids, p, duration=1.0)], 0.01, 0.1)
        assert nbytes[0] > 0 and kernel[0] >= 32
        assert (levels[0] > 1) == (model == "turing")   # Turing reads rows written in the same step
        off, ids = default_graph(65537, 1)
        with pytest.raises(E.DenseError, match="error 4"):
            E.plan(model, [E.ParameterSet(off, ids, p, duration=1.0)], 0.01, 0.1)


def test_perturbation_factors_resize_the_rings():
    """-b factors scale the delays that size DENSE's rings (S = (int)(max
    delay x (1 + factor) / dt) + 2).  mh13 is read at delay 0.805 min
    (k = 0, so lag S - 1): a factor of 0.6 on ph13_synthesis takes its S
    from 82 to 130 rows (as in DENSE, checked on the oracle), which doubles
    the register kernel's power-of-two staging of mh13 from 128 to 256
    rows; the plan grows by exactly those rows."""
    from oracle.pyoracle import load_oracle
    L = E.load("her_model_2014")
    p = workloads.template_params()
    off, ids = default_graph(20, 4)
    pert = np.zeros(L.num_reactions)
    pert[L.reactions.index("ph13_synthesis")] = 0.6
    mh13 = L.species.index("mh13")
    O = load_oracle("her_model_2014")
    S0 = O.create(off, ids, np.tile(p, (20, 1)), p, None, 0.01).ring_sizes()[0]
    S1 = O.create(off, ids, np.tile(p, (20, 1)), p, None, 0.01, pert).ring_sizes()[0]
    assert S0[mh13] == 82 and S1[mh13] == 130
    assert [S0[i] for i in range(14) if i != mh13] == [S1[i] for i in range(14) if i != mh13]
    b0, _, _ = E.plan("her_model_2014", [E.ParameterSet(off, ids, p, duration=1.0)], 0.01, 0.1)
    b1, _, _ = E.plan("her_model_2014", [E.ParameterSet(off, ids, p, duration=1.0, perturb=pert)], 0.01, 0.1)
    assert b1[0] - b0[0] == 8 * (256 - 128) * 20
