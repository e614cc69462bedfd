"""dense_simulate_noalloc, the entry point for callers that may not
allocate device memory (a framework that owns the GPU's memory pool, or a
loop that must not call cudaMalloc after start-up).

Called through the C ABI twice in a row on the same batch (sets with one
parameter row, sets with per-cell parameter matrices, and a set with a NaN
rate that DENSE would reject); both results must equal, bit for bit (the
FP64 tolerance of every other test here), the final state and the status
words the allocating entry points (dense_engine_create / run / read_state /
status) give.  This file is collected after the engine, CLI, mixed and
surrogate tests, so a failure here comes after all of them have run.
"""

import ctypes as C

import numpy as np
import pytest

from dense_b200 import engine as E
from dense_b200 import workloads
from dense_b200.tissue import default_graph

pytestmark = pytest.mark.gpu


def _inputs():
    P = workloads.log_uniform_params(5, seed=21)
    off, ids = default_graph(48, 4)
    sets = [E.ParameterSet(off, ids, P[i], duration=20.0) for i in range(5)]
    # two sets with per-cell parameter matrices, one after the other (each
    # goes through the shared staging area into the [param][cell] layout)
    sets.append(workloads.perturbed_set(cells=40, width=5, duration=15.0, seed=22))
    sets.append(workloads.perturbed_set(cells=24, width=4, duration=12.0, seed=23))
    # a set DENSE would reject (a NaN rate): its status word must say so
    bad = P[0].copy()
    bad[3] = np.nan
    sets.append(E.ParameterSet(off, ids, bad, duration=5.0))
    return sets


def _descs(L, sets):
    arr = (E._SetDesc * len(sets))()
    for i, s in enumerate(sets):
        arr[i].num_cells = s.num_cells
        arr[i].nbr_offsets = E._ip(s.nbr_offsets)
        arr[i].nbr_ids = E._ip(s.nbr_ids)
        arr[i].set_params = E._dp(s.set_params)
        arr[i].cell_params = E._dp(s.cell_params)
        arr[i].init_conc = E._dp(s.init_conc)
        arr[i].perturb = E._dp(s.perturb)
        arr[i].duration = s.duration
    return arr


def _noalloc(L, sets, run):
    f = L.lib.dense_simulate_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(E._RunDesc), C.c_int, C.POINTER(E._SetDesc), C.POINTER(C.c_double),
                  C.POINTER(C.c_int32), C.c_void_p]
    total = sum(L.num_species * s.num_cells for s in sets)
    out = np.full(total, np.nan)
    status = np.full(len(sets), -1, np.int32)
    rc = f(C.byref(run), len(sets), _descs(L, sets), out.ctypes.data_as(C.POINTER(C.c_double)),
           status.ctypes.data_as(C.POINTER(C.c_int32)), None)
    return rc, out, status


def test_noalloc_matches_allocating_entry_point_twice():
    L = E.load("her_model_2014")
    sets = _inputs()
    b = E.Batch(L, sets, 0.01, 0.1, [])
    b.run()
    b.sync()
    want = np.concatenate([b.state(i).ravel() for i in range(len(sets))])
    want_status = b.status()
    assert (want_status[:-1] == 0).all() and want_status[-1] == 2  # DENSE_SET_NAN_PARAM
    b.close()
    run = E._RunDesc(E.FP64, 0.01, 0.1, 0, None, 0)
    for _ in range(2):
        rc, got, status = _noalloc(L, sets, run)
        assert rc == 0
        assert np.array_equal(status, want_status)
        assert np.array_equal(got, want)


def test_noalloc_rejects_a_batch_beyond_its_scratch():
    L = E.load("her_model_2014")
    off, ids = default_graph(200, 4)
    p = workloads.template_params()
    run = E._RunDesc(E.FP64, 0.01, 0.1, 0, None, 0)
    # 64 sets of 200 cells need about 20 MiB of descriptors, parameters,
    # state and history: more than the 16 MiB array
    rc, _, _ = _noalloc(L, [E.ParameterSet(off, ids, p, duration=1.0) for _ in range(64)], run)
    assert rc == 5  # DENSE_ERR_SCRATCH_TOO_SMALL
    # more than 64 sets
    small_off, small_ids = default_graph(4, 2)
    rc, _, _ = _noalloc(L, [E.ParameterSet(small_off, small_ids, p, duration=1.0) for _ in range(65)], run)
    assert rc == 5
