"""The benchmark configurations' seeded synthetic inputs match their
descriptions: the one-set configuration (per-cell, per-parameter factors in
[0.95, 1.05]) and the batched one (per-set factors exp(U(ln 1/2, ln 2)),
zero parameters staying zero), on DENSE's default 200-cell tissue."""

import numpy as np

from dense_b200 import workloads
from dense_b200.tissue import default_graph


def test_one_set_configuration():
    s = workloads.perturbed_set(cells=200, width=4, duration=600.0, seed=1)
    t = workloads.template_params()
    assert s.num_cells == 200 and s.duration == 600.0 and s.cell_params.shape == (200, t.size)
    nz = t > 0
    r = s.cell_params[:, nz] / t[nz]
    assert (r >= 0.95).all() and (r <= 1.05).all() and r.std() > 0.02
    assert (s.cell_params[:, ~nz] == 0).all()
    off, ids = default_graph(200, 4)
    assert np.array_equal(s.nbr_offsets, off) and np.array_equal(s.nbr_ids, ids)
    # 100 cells with 4 out-neighbours and 100 with 5 (cell 0 -> 3, 196, 197, 199)
    deg = np.diff(off)
    assert (deg == 4).sum() == 100 and (deg == 5).sum() == 100
    assert ids[off[0]:off[1]].tolist() == [3, 196, 197, 199]
    again = workloads.perturbed_set(cells=200, width=4, duration=600.0, seed=1)
    assert np.array_equal(again.cell_params, s.cell_params)


def test_batched_configuration():
    sets = workloads.log_uniform_sets(64, cells=200, width=4, duration=1200.0, seed=2)
    t = workloads.template_params()
    nz = t > 0
    F = np.array([s.set_params[nz] / t[nz] for s in sets])
    assert (F >= 0.5).all() and (F <= 2.0).all()
    logf = np.log(F)
    assert abs(logf.mean()) < 0.05 and abs(logf.std() - np.log(2.0) / np.sqrt(3.0)) < 0.03   # U(-ln2, ln2)
    assert all((s.set_params[~nz] == 0).all() and s.cell_params is None and s.duration == 1200.0 for s in sets)
    assert len({s.set_params.tobytes() for s in sets}) == 64
