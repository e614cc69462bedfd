"""The surrogate experiment on one GPU, end to end:

  1. draw seeded log-uniform +-4x candidates of her_model_2014 and simulate
     a training set and a held-out set with the FP64 engine (features of
     dense_b200.search);
  2. train the MLP surrogate on the tensor-core kernels;
  3. report the held-out feature error against the FP64 simulation;
  4. surrogate-screened search on fresh candidates (top 1% re-simulated in
     FP64) against plain GPU search on the same candidates (a random sample
     simulated, rate extrapolated per candidate);
  5. a few SRES generations with and without the surrogate in front of the
     scorer.

Prints one JSON object.  Usage:
  python -m dense_b200.search_run [--train N] [--test N] [--candidates N]
      [--minutes M] [--resim-minutes R[,R2...]] [--cells C] [--epochs E]
      [--ensemble K] [--generations G] [--extrapolate N[,N2...]]
      [--refine K [--refine-pool N] [--refine-rounds R]] [--data-cache FILE]

--minutes is the horizon of the training and held-out simulations (the
features' window is 0-60 min, and the first 60 minutes of a run do not
depend on what follows); --resim-minutes the horizons at which the search
simulates its candidates -- the screened survivors and the plain-search
sample alike -- the first one reported as "search", each one also under
"search_by_horizon" with the same trained network and candidates (default
1200 min, the configuration's horizon, and 60 min beside it).

Under torchrun (one process per GPU) steps 1, 2 and 4 shard: each rank
simulates its share of the training candidates, the surrogate trains
data-parallel (gradients averaged each step over NCCL), and the screening
scores each rank's share of the candidates, merges the global top 1% and
re-simulates it spread over the ranks (dense_b200.distributed); the
candidates then come from chunked seeded streams; the plain-search
baseline and SRES stay single-GPU (rank 0 reports).
"""

import argparse
import json
import os
import sys
import time

import numpy as np

from . import search as S


def with_one_time_cost(res, candidates=None):
    """The screened search's rate charged with the surrogate's one-time cost
    (training simulations and training), crediting the sets the training
    simulations accepted, and its gain over plain search; None where the
    run has no plain rate.  With `candidates` other than the run's, the
    same figures for a search of that many candidates per trained network,
    scaled from the run's measured parts: ranking, re-simulation and
    accepted sets grow with the candidates, the one-time cost does not."""
    srch, data = res["search"], res["data"]
    scale = 1.0 if candidates is None else candidates / float(srch["candidates"])
    seconds = data["seconds"] + res["training_s"] + scale * (srch["inference_s"] + srch["resimulation_s"])
    accepted = scale * srch["accepted_screened"] + data["accepted_fraction"] * data["train_sets"]
    rate = accepted / seconds
    plain = srch["accepted_per_s_plain"]
    out = {"accepted_per_s": rate, "gain": rate / plain if plain > 0 else None, "seconds": seconds}
    if candidates is not None:
        out["candidates"] = candidates
    return out


def load_or_simulate(a, sim, log):
    """Training and held-out candidates and their FP64 features; with
    --data-cache, read from that file when it exists (the recorded
    simulation seconds are the original run's) and written otherwise."""
    import pickle
    if a.data_cache and os.path.exists(a.data_cache):
        with open(a.data_cache, "rb") as f:
            return pickle.load(f), True
    P_train = S.draw_candidates(a.train, a.seed)
    F_train = S.simulate_features(P_train, log=log, **sim)
    P_test = S.draw_candidates(a.test, a.seed + 1)
    F_test = S.simulate_features(P_test, log=log, **sim)
    data = (P_train, F_train, P_test, F_test)
    if a.data_cache:
        with open(a.data_cache, "wb") as f:
            pickle.dump(data, f)
    return data, False


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=200000)
    ap.add_argument("--test", type=int, default=4096)
    ap.add_argument("--candidates", type=int, default=1000000)
    ap.add_argument("--keep", type=float, default=0.01)
    ap.add_argument("--plain-sample", type=int, default=4096)
    ap.add_argument("--minutes", type=float, default=60.0,
                    help="simulated minutes of the training data (the feature window is 0-60)")
    ap.add_argument("--resim-minutes", default="1200,60",
                    help="simulated minutes of the search's simulations, comma-separated")
    ap.add_argument("--cells", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--ensemble", type=int, default=4, help="networks averaged by the surrogate")
    ap.add_argument("--generations", type=int, default=3)
    ap.add_argument("--seed", type=int, default=100)
    ap.add_argument("--refine", type=int, default=50000,
                    help="candidates the first network ranks best in a fresh pool, simulated and added to the "
                         "training set before the networks are trained again (0: no refinement)")
    ap.add_argument("--refine-pool", type=int, default=2000000)
    ap.add_argument("--refine-rounds", type=int, default=3)
    ap.add_argument("--extrapolate", default="58000000",
                    help="candidate counts for the charged gain scaled from the measured run, comma-separated")
    ap.add_argument("--data-cache", default=None,
                    help="file holding the simulated training and held-out sets (read if present, else written)")
    a = ap.parse_args(argv)
    log = lambda m: print(m, file=sys.stderr, flush=True)  # noqa: E731
    if int(os.environ.get("WORLD_SIZE", "1")) > 1:
        return sharded(a, log)
    sim = dict(minutes=a.minutes, cells=a.cells, width=4)
    res = {"config": vars(a)}
    t0 = time.perf_counter()
    (P_train, F_train, P_test, F_test), cached = load_or_simulate(a, sim, log)
    res["data_cached"] = cached
    res["data"] = {"train_sets": a.train, "test_sets": a.test, "seconds": F_train["seconds"] + F_test["seconds"],
                   "cell_steps_per_s": (F_train["cell_steps"] + F_test["cell_steps"]) /
                                       (F_train["seconds"] + F_test["seconds"]),
                   "oscillating_fraction": float(F_train["oscillates"].mean()),
                   "accepted_fraction": float(S.accepted(F_train).mean())}
    t1 = time.perf_counter()
    net = S.train_surrogate(P_train, F_train, epochs=a.epochs, batch=2048, seed=a.seed, log=log,
                            ensemble=a.ensemble)
    res["training_s"] = time.perf_counter() - t1
    res["refine"] = []
    if a.refine > 0 and a.refine_rounds > 0:
        # refinement rounds: the current networks rank a fresh pool, its
        # best `refine` candidates are simulated and join the training set
        # (they lie where the search looks), and the networks are trained
        # again on everything; all of it counts in the one-time cost
        t2 = time.perf_counter()
        train = lambda P, F: S.train_surrogate(P, F, epochs=a.epochs, batch=2048, seed=a.seed, log=log,  # noqa
                                               ensemble=a.ensemble)
        net, P_train, F_train, rounds = S.refine(net, P_train, F_train, train, a.refine_rounds, a.refine,
                                                 a.refine_pool, a.seed + 3,
                                                 simulate=lambda P: S.simulate_features(P, log=log, **sim))
        sim_s = sum(r["seconds"] for r in rounds)
        res["refine"] = [{k: v for k, v in r.items() if k != "kept"} for r in rounds]
        res["training_s"] += time.perf_counter() - t2 - sim_s
        res["data"]["train_sets"] = len(P_train)
        res["data"]["seconds"] += sim_s
        res["data"]["accepted_fraction"] = float(S.accepted(F_train).mean())
    res["held_out_error"] = S.feature_errors(net, P_test, F_test)
    res["search_by_horizon"] = {}
    for k, m in enumerate(float(x) for x in str(a.resim_minutes).split(",")):
        r = S.screened_search(net, a.candidates, a.seed + 2, keep=a.keep, plain_sample=a.plain_sample,
                              sim_kwargs=dict(sim, minutes=m), log=log)
        r["minutes"] = m
        r["with_one_time_cost"] = with_one_time_cost(dict(res, search=r))
        if a.extrapolate:
            r["with_one_time_cost_scaled"] = [with_one_time_cost(dict(res, search=r), int(float(c)))
                                              for c in str(a.extrapolate).split(",")]
        res["search_by_horizon"]["%g" % m] = r
        if k == 0:
            res["search"] = r
            res["search_with_one_time_cost"] = r["with_one_time_cost"]
    if a.generations > 0:
        fit = lambda X: S.search_fitness(S.simulate_features(S.decode(X), **sim))  # noqa: E731
        pred = lambda X: S.predicted_score(net.predict(X.astype(np.float32)))  # noqa: E731
        d = len(S.active_params())
        for name, kw in (("plain", {}), ("screened", {"surrogate": pred, "screen": 8})):
            es = S.SRES(d, fit, mu=16, lam=128, seed=a.seed, **kw)
            best = [float(np.min(es.f))]
            for _ in range(a.generations):
                best.append(es.step())
            res["sres_" + name] = {"best_fitness_per_generation": best, "simulations": es.evaluations}
    res["total_s"] = time.perf_counter() - t0
    print(json.dumps(res))


def sharded(a, log):
    import datetime
    import torch
    import torch.distributed as dist
    from . import distributed as D
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    rank, world = dist.get_rank(), dist.get_world_size()
    sim = dict(minutes=a.minutes, cells=a.cells, width=4, device=local)
    res = {"config": vars(a), "ranks": world}
    t0 = time.perf_counter()
    lo, hi = D.shard_range(a.train, rank, world)
    P = D.candidate_range(lo, hi, a.seed, S._draw_rows)
    F = S.simulate_features(P, log=log if rank == 0 else None, **sim)
    t = torch.tensor([F["seconds"]], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    res["data"] = {"train_sets": a.train, "seconds_max_over_ranks": float(t.item())}
    t1 = time.perf_counter()
    net = S.train_surrogate(P, F, epochs=a.epochs, batch=2048, seed=a.seed, log=log if rank == 0 else None,
                            group=dist.group.WORLD, device=local, ensemble=a.ensemble)
    res["training_s"] = time.perf_counter() - t1
    res["search"] = S.screened_search_sharded(net, a.candidates, a.seed + 2, keep=a.keep,
                                              group=dist.group.WORLD,
                                              sim_kwargs=dict(sim, minutes=float(str(a.resim_minutes).split(",")[0])),
                                              log=log if rank == 0 else None)
    res["total_s"] = time.perf_counter() - t0
    if rank == 0:
        print(json.dumps(res))
    dist.destroy_process_group()


if __name__ == "__main__":
    main()
