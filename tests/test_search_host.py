"""Host-side facts the surrogate search relies on, checked on the oracle
(bit-exact with the engine, pinned against DENSE)."""

import numpy as np

from dense_b200 import search as S, workloads
from dense_b200.tissue import default_graph


def test_features_do_not_depend_on_the_horizon_past_the_window():
    """The search's Oscillation features over [0, 60) are identical whether
    the simulation stops at 60 minutes or runs on to 120, so the features
    are simulated to the window's end only."""
    from oracle.pyoracle import load_oracle
    O = load_oracle("her_model_2014")
    P = S.draw_candidates(4, 9)
    off, ids = default_graph(24, 4)
    mh1 = workloads.her_species("mh1")
    for p in P:
        res = []
        for minutes in (60.0, 120.0):
            sim = O.create(off, ids, np.tile(p, (24, 1)), p, None, 0.01)
            sim.add_oscillation(mh1, 0, 24, 0.0, 60.0, 4.0, 0.1)
            sim.run(minutes, 0.1)
            res.append(sim.oscillation(0))
        for k in ("amps", "pers", "avg_peak", "ncrit", "samples"):
            assert np.array_equal(np.asarray(res[0][k]), np.asarray(res[1][k]), equal_nan=True), k
