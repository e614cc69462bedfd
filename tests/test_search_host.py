"""Host-side parts of the surrogate search: the horizon fact it relies on
(checked on the oracle, bit-exact with the engine), the parameter encoding,
synchrony, acceptance and fitness, and the evolution strategy."""

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


def test_encode_decode_round_trip():
    rng = np.random.Generator(np.random.PCG64(3))
    X = rng.uniform(-1, 1, size=(64, len(S.active_params())))
    assert np.allclose(S.encode(S.decode(X)), X, atol=1e-6)
    P = S.draw_candidates(256, 4)
    E = S.encode(P)
    assert E.shape == (256, 44) and np.abs(E).max() <= 1.0 + 1e-6
    # parameters that are zero in the template stay zero
    zero = np.setdiff1d(np.arange(P.shape[1]), S.active_params())
    assert (S.decode(X)[:, zero] == 0).all()


def test_synchrony_known_answers_on_the_host():
    t = np.linspace(0, 20, 400)[:, None]
    assert abs(S.synchrony(np.sin(t) * np.ones((1, 8))) - 1.0) < 1e-12
    assert abs(S.synchrony(np.concatenate([np.sin(t), -np.sin(t)], 1)) + 1.0) < 1e-12
    # a constant cell is left out; fewer than two varying cells: undefined
    with_flat = np.concatenate([np.sin(t), np.sin(t), np.full_like(t, 3.0)], 1)
    assert abs(S.synchrony(with_flat) - 1.0) < 1e-12
    assert np.isnan(S.synchrony(np.concatenate([np.sin(t), np.full_like(t, 3.0)], 1)))
    # quarter-period shift: uncorrelated over whole periods
    q = np.linspace(0, 2 * np.pi * 10, 4000, endpoint=False)[:, None]
    assert abs(S.synchrony(np.concatenate([np.sin(q), np.cos(q)], 1))) < 1e-9


def test_acceptance_targets_and_fitness():
    F = {"period": np.array([30.0, 33.0, 33.5, np.nan, 28.0]),
         "amplitude": np.array([60.0, 50.0, 80.0, 90.0, 10.0]),
         "synchrony": np.array([0.9, np.nan, 0.1, 0.2, 0.3]),
         "oscillates": np.array([1.0, 1.0, 1.0, 0.0, 1.0], np.float32)}
    assert S.accepted(F).tolist() == [True, True, False, False, False]
    T, M = S.targets(F)
    assert T.shape == (5, 5) and np.isfinite(T).all()
    assert M[:, 0].tolist() == [1, 1, 1, 0, 1] and M[1, 2] == 0 and M[:, 4].tolist() == [1] * 5
    f = S.search_fitness(F)
    assert f[0] == 0.0 and f[1] == 1.0 and f[3] == 1e3
    assert abs(f[4] - (2.0 / 3.0 + 0.8)) < 1e-12


def _sphere(X):
    return ((X - 0.3) ** 2).sum(axis=1)


def test_sres_converges_on_a_smooth_function():
    """The evolution strategy alone (no simulator) on a shifted sphere in the
    search box: steady progress, offspring inside [-1, 1], evaluations
    counted, the same seed giving the same run."""
    es = S.SRES(10, _sphere, mu=15, lam=100, seed=4)
    f0 = float(es.f.min())
    best = [es.step() for _ in range(200)]
    # the step sizes adapt through exponential smoothing (alpha 0.2), so
    # progress is steady rather than fast: ~1.5 -> ~2e-5 here
    assert best[59] < 0.1 * f0 and best[199] < 0.01 * best[59] and best[199] < 1e-4
    assert np.abs(es.x).max() <= 1.0 and es.evaluations == 100 * 201
    es2 = S.SRES(10, _sphere, mu=15, lam=100, seed=4)
    assert [es2.step() for _ in range(200)] == best


def test_sres_gains_from_a_surrogate():
    """With a surrogate ranking 8x lambda offspring (here an exact one) the
    strategy reaches a lower fitness for the same number of simulated
    evaluations."""
    plain = S.SRES(20, _sphere, mu=15, lam=100, seed=6)
    screened = S.SRES(20, _sphere, mu=15, lam=100, seed=6, surrogate=lambda X: -_sphere(X), screen=8)
    for _ in range(25):
        bp, bs = plain.step(), screened.step()
    assert plain.evaluations == screened.evaluations
    assert bs < 0.5 * bp


def test_gain_with_one_time_cost():
    """The screened rate charged with training simulations and training,
    on the figures of a recorded 10M-candidate run (200k training sets)."""
    from dense_b200.search_run import with_one_time_cost
    res = {"data": {"seconds": 69.686775528, "train_sets": 200000, "accepted_fraction": 0.03212},
           "training_s": 49.90117416199999,
           "search": {"candidates": 10000000, "inference_s": 0.4650351440000122,
                      "resimulation_s": 31.993933156999987, "accepted_screened": 49294,
                      "accepted_per_s_plain": 95.1213437156791}}
    r = with_one_time_cost(res)
    assert abs(r["accepted_per_s"] - 366.45) < 0.1 and abs(r["gain"] - 3.85) < 0.01
    # scaled to 58M candidates: 5.8x the search parts, the same one-time cost
    r58 = with_one_time_cost(res, 58000000)
    want = (5.8 * 49294 + 0.03212 * 200000) / (69.686775528 + 49.90117416199999 + 5.8 * (0.4650351440000122 +
                                                                                     31.993933156999987))
    assert abs(r58["accepted_per_s"] - want) < 1e-9 and r58["candidates"] == 58000000
    assert abs(with_one_time_cost(res, 10000000)["gain"] - r["gain"]) < 1e-12
    res["search"]["accepted_per_s_plain"] = 0.0
    assert with_one_time_cost(res)["gain"] is None


def test_merge_features_concatenates_in_order():
    from dense_b200.search import merge_features
    a = {"period": np.array([1.0, 2.0]), "status": np.array([0, 1], np.int32), "seconds": 1.5, "cell_steps": 10}
    b = {"period": np.array([3.0]), "status": np.array([2], np.int32), "seconds": 0.5, "cell_steps": 4}
    m = merge_features(a, b)
    assert m["period"].tolist() == [1.0, 2.0, 3.0] and m["status"].tolist() == [0, 1, 2]
    assert m["seconds"] == 2.0 and m["cell_steps"] == 14


def test_refinement_rounds_grow_the_training_set_with_the_best_ranked():
    """Each round ranks a fresh pool, simulates its `keep` best and trains
    on everything so far (fakes for the network, the scorer and the
    simulator; the pools differ per round)."""
    calls = []

    def draw(n, seed):
        return np.random.Generator(np.random.PCG64(seed)).uniform(size=(n, 3))

    def score(net, P):
        return P[:, 0] * net        # the "network" is a weight on the first column

    def simulate(P):
        per = 30.0 + 10.0 * (1.0 - P[:, 0])
        return {"period": per, "amplitude": np.full(len(P), 60.0), "seconds": 0.5, "cell_steps": len(P)}

    def train(P, F):
        calls.append((len(P), len(F["period"])))
        return 1.0 + len(calls)

    P0 = np.zeros((10, 3))
    F0 = {"period": np.full(10, np.nan), "amplitude": np.full(10, np.nan), "seconds": 1.0, "cell_steps": 10}
    net, P, F, rec = S.refine(2.0, P0, F0, train, rounds=3, keep=5, pool_size=100, seed=7, score=score,
                              simulate=simulate, draw=draw)
    assert calls == [(15, 15), (20, 20), (25, 25)] and net == 4.0
    assert len(P) == 25 and F["seconds"] == 1.0 + 3 * 0.5 and F["cell_steps"] == 25
    for r, k in enumerate(rec):
        pool = draw(100, 7 + r)
        best = set(np.argsort(-pool[:, 0])[:5].tolist())
        assert set(k["kept"].tolist()) == best
        assert set(map(tuple, P[10 + 5 * r:15 + 5 * r])) == set(map(tuple, pool[k["kept"]]))
    # the best of each pool have period within 30 +- 3 (first column > 0.7) and are accepted
    assert all(k["accepted_fraction_of_simulated"] > 0.5 for k in rec)
