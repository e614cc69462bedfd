"""Parameter search for her_model_2014 on the batched FP64 engine, with the
MLP surrogate in front of the simulator.

DENSE's search (search/sres.hpp:202-265, sres.cpp:328-349) evolves a
population with SRES and scores each candidate by simulating it.  Here a
whole population is simulated as one engine batch, and the surrogate
(dense_b200.surrogate) ranks candidates before any simulation: only the
candidates it ranks best are simulated, and only the FP64 engine's
results decide acceptance.

Features of one simulated set (200 cells by default), all over the first
`window` minutes -- the window of DENSE's own oscillation test
(test/her_model_2014/analyses.xml).  DENSE passes delays in minutes where
its history expects steps (sim/base.hpp:406-422), so the effective delays
are ~100x shorter than the parameters say and the her clock is a transient
that settles within ~100 simulated minutes; later windows show no
oscillation:
  * period    -- mean over cells of mh1's OscillationAnalysis period;
  * amplitude -- mean over cells of mh1's OscillationAnalysis amplitude;
  * synchrony -- mean pairwise Pearson correlation of mh1 across cells
                 (DENSE has no synchrony measure;
                 CorrelationAnalysis::pearson_correlate is declared but never
                 defined, measurement/oscillation.hpp:119-136);
  * oscillates -- finite period and amplitude above OSC_AMP.
A candidate is accepted when its period is TARGET_PERIOD +- PERIOD_TOL and
its amplitude at least AMP_MIN (fixed here at 50, about twice the
template's amplitude).
"""

import math
import time

import numpy as np

from . import engine as E
from . import workloads
from .tissue import default_graph

TARGET_PERIOD = 30.0
PERIOD_TOL = 3.0
AMP_MIN = 50.0
OSC_AMP = 1.0
SPREAD = 4.0


def template():
    return workloads.template_params("her_model_2014")


def active_params():
    """Indices of the template's non-zero parameters (the search space)."""
    return np.nonzero(template())[0]


def draw_candidates(n, seed, spread=SPREAD):
    """Log-uniform +-spread x around the template, [n][NP]."""
    return workloads.log_uniform_params(n, 1.0 / spread, spread, seed=seed)


def encode(P, spread=SPREAD):
    """Surrogate inputs: log(p / template) / log(spread) of the active
    parameters, in [-1, 1] for the search box."""
    t = template()
    idx = active_params()
    return (np.log(P[:, idx] / t[idx]) / math.log(spread)).astype(np.float32)


def synchrony(traj):
    """Mean pairwise Pearson correlation across cells of traj [samples][cells]
    (cells with a constant trace are left out), by
    sum_{i != j} <z_i, z_j> = |sum_i z_i|^2 - sum_i |z_i|^2 on unit z_i."""
    x = traj - traj.mean(axis=0, keepdims=True)
    nrm = np.sqrt((x * x).sum(axis=0))
    ok = nrm > 1e-12 * (1.0 + np.abs(traj).max())
    n = int(ok.sum())
    if n < 2:
        return float("nan")
    z = x[:, ok] / nrm[ok]
    s = z.sum(axis=1)
    return float(((s * s).sum() - n) / (n * (n - 1)))


def _kernels(device):
    """The surrogate library's launchers on `device` (one per device)."""
    from .surrogate import Kernels
    k = _KERNELS.get(device)
    if k is None:
        k = _KERNELS[device] = Kernels(device)
    return k


_KERNELS = {}


def synchrony_batch(X, counts):
    """synchrony() of every set at once on the GPU (one CTA per set,
    csrc/surrogate/features.cu): X [sets][samples][cells] (a float64 CUDA
    tensor, cells contiguous; rows past a set's count are ignored), counts
    [sets]; float64 numpy array out."""
    import torch
    k = _kernels(X.device.index or 0)
    cnt = torch.as_tensor(np.asarray(counts, np.int32), device=X.device)
    out = torch.empty(X.shape[0], dtype=torch.float64, device=X.device)
    k.synchrony(X, cnt, out)
    return out.cpu().numpy()


def simulate_features(P, minutes=None, cells=200, width=4, window=60.0, batch=4096, device=0,
                      precision=E.FP64, log=None):
    """Simulates every row of P (one set each) and returns its features.

    Every feature is taken over [0, window), and the first `window` minutes
    of a forward simulation do not depend on what follows, so the horizon
    defaults to the window's end (`minutes`=None); a longer horizon gives
    the same features at a higher cost."""
    minutes = window if minutes is None else minutes
    off, ids = default_graph(cells, width)
    mh1 = workloads.her_species("mh1")
    n = P.shape[0]
    out = {k: np.full(n, np.nan) for k in ("period", "amplitude", "synchrony")}
    out["status"] = np.zeros(n, np.int32)
    t0 = time.perf_counter()
    cell_steps = 0
    for s in range(0, n, batch):
        rows = P[s:s + batch]
        sets = [E.ParameterSet(off, ids, p, duration=minutes) for p in rows]
        an = [E.Analysis.oscillation(mh1, 0, cells, 0.0, window, 4.0, 0.1),
              E.Analysis.trajectory(mh1, 0, cells, 0.0, window)]
        b = E.Batch("her_model_2014", sets, 0.01, 0.1, an, precision=precision, device=device)
        b.run()
        b.sync()
        st = b.status()
        cell_steps += b.info()["total_cell_steps"]
        # every set's results in two strided copies and one device copy
        amps, pers = b.oscillation_all(0)
        with np.errstate(invalid="ignore"):
            for key, v in (("period", pers[:, 0, :]), ("amplitude", amps[:, 0, :])):
                # per set: the mean of the non-NaN cells, if any cell is finite
                num = ~np.isnan(v)
                tot = np.where(num, v, 0.0).sum(1)
                mean = tot / np.maximum(num.sum(1), 1)
                out[key][s:s + len(rows)] = np.where(np.isfinite(v).any(1), mean, np.nan)
        traj, cnt = b.trajectory_device(1)
        out["synchrony"][s:s + len(rows)] = synchrony_batch(traj[:, :, 0, :], cnt)
        del traj
        out["status"][s:s + len(rows)] = st
        b.close()
        if log:
            log("simulated %d / %d sets" % (min(s + batch, n), n))
    out["oscillates"] = (np.isfinite(out["period"]) & (np.nan_to_num(out["amplitude"]) > OSC_AMP)).astype(np.float32)
    out["seconds"] = time.perf_counter() - t0
    out["cell_steps"] = cell_steps
    return out


def accepted(F):
    per, amp = F["period"], F["amplitude"]
    with np.errstate(invalid="ignore"):
        return np.isfinite(per) & (np.abs(per - TARGET_PERIOD) <= PERIOD_TOL) & (np.nan_to_num(amp) >= AMP_MIN)


def merge_features(*Fs):
    """One feature dict from several simulate_features results: the per-set
    arrays concatenated in order, seconds and cell-steps summed."""
    out = {}
    for key in Fs[0]:
        if key in ("seconds", "cell_steps"):
            out[key] = sum(F[key] for F in Fs)
        else:
            out[key] = np.concatenate([np.asarray(F[key]) for F in Fs])
    return out


def refine(net, P_train, F_train, train, rounds, keep, pool_size, seed, score=None, simulate=None, draw=None):
    """Refinement rounds (active learning): per round, the current networks
    rank a fresh pool of `pool_size` candidates (seed + round), the best
    `keep` (fewer than `pool_size`) are simulated and join the training
    set, and `train(P, F)` makes new networks from everything.  Returns the final networks, the grown
    training set and one record per round (pool, simulated, simulation
    seconds, accepted share, indices kept).  score / simulate / draw
    default to score_candidates / simulate_features / draw_candidates."""
    score = score or score_candidates
    simulate = simulate or simulate_features
    draw = draw or draw_candidates
    records = []
    for r in range(rounds):
        pool = draw(pool_size, seed + r)
        top = np.argpartition(-score(net, pool), keep)[:keep]
        F_new = simulate(pool[top])
        P_train = np.concatenate([P_train, pool[top]])
        F_train = merge_features(F_train, F_new)
        net = train(P_train, F_train)
        records.append({"pool": pool_size, "simulated": keep, "seconds": F_new["seconds"],
                        "accepted_fraction_of_simulated": float(accepted(F_new).mean()), "kept": np.sort(top)})
    return net, P_train, F_train, records


def targets(F):
    """Surrogate targets [n][5]: log period, log amplitude, synchrony, the
    oscillation indicator and the acceptance indicator; and their mask
    (feature defined)."""
    with np.errstate(invalid="ignore", divide="ignore"):
        T = np.stack([np.log(F["period"]), np.log(F["amplitude"]), F["synchrony"], F["oscillates"],
                      accepted(F).astype(np.float64)], 1)
    osc = F["oscillates"] > 0.5
    one = np.ones_like(osc)
    M = np.stack([osc, osc, np.isfinite(F["synchrony"]), one, one], 1).astype(np.float32)
    M = M * np.isfinite(T)
    return np.nan_to_num(T).astype(np.float32), M.astype(np.float32)


class Surrogate:
    """The trained networks behind one predict(): outputs trained
    standardised (minus their mean over the rows where they are defined,
    over their standard deviation there; mu 0 and sd 1 leave an output as
    it is) are mapped back on prediction; with several networks (an
    ensemble of different initial weights and batch orders) their outputs
    are averaged."""

    def __init__(self, nets, mu, sd):
        self.nets, self.mu, self.sd = nets, np.asarray(mu, np.float32), np.asarray(sd, np.float32)
        self.dev = nets[0].dev

    def predict(self, X):
        y = sum(n.predict(X) for n in self.nets) / len(self.nets)
        return y * self.sd + self.mu

    def predict_device(self, x):
        import torch
        y = sum(n.predict_device(x) for n in self.nets) / len(self.nets)
        return y * torch.as_tensor(self.sd, device=y.device) + torch.as_tensor(self.mu, device=y.device)


def train_surrogate(P, F, epochs=30, batch=4096, seed=0, lr=1e-3, log=None, group=None, device=0, ensemble=1,
                    standardize_indicators=False):
    """The MLP surrogate on (P, F): `ensemble` networks trained on
    standardised regression targets (the 0/1 indicators too with
    `standardize_indicators`, which weighs the rare acceptances up); with a
    process group, data-parallel over the ranks' shards (gradients averaged
    every step)."""
    from .surrogate import MLP, fit_concurrently
    X = encode(P)
    T, M = targets(F)
    mu = np.zeros(T.shape[1], np.float32)
    sd = np.ones(T.shape[1], np.float32)
    for j in range(T.shape[1] if standardize_indicators else 3):
        on = M[:, j] > 0
        if on.sum() > 1:
            mu[j] = float(T[on, j].mean())
            sd[j] = max(1e-6, float(T[on, j].std()))
    if group is not None:
        # the same scaling on every rank: the mean of the ranks' statistics
        import torch
        import torch.distributed as dist
        t = torch.as_tensor(np.concatenate([mu, sd]), dtype=torch.float64)
        if dist.get_backend(group) == "nccl":
            t = t.cuda(device)
        dist.all_reduce(t, group=group)
        t = (t / dist.get_world_size(group)).cpu().numpy().astype(np.float32)
        mu, sd = t[:T.shape[1]], t[T.shape[1]:]
    Ts = ((T - mu) / sd) * M
    nets = [MLP(X.shape[1], T.shape[1], seed=seed + 1000 * k, lr=lr, group=group, device=device)
            for k in range(ensemble)]
    b = min(batch, (X.shape[0] // 128) * 128)
    if group is None and ensemble > 1:
        # the ensemble's networks train at once, one CUDA stream each
        fit_concurrently(nets, X, Ts, M, [seed + 1000 * k for k in range(ensemble)], epochs=epochs, batch=b,
                         log=log)
    else:
        for k, net in enumerate(nets):
            net.fit(X, Ts, M, epochs=epochs, batch=b, seed=seed + 1000 * k, log=log)
    return Surrogate(nets, mu, sd)


REGION_WEIGHT = 0.1   # weight of the predicted features' closeness to the acceptance region
AMP_RAMP = 0.1        # log-amplitude width over which the amplitude term rises from 0 to 1


def _region_terms(log_per, log_amp, p_osc):
    """Closeness of the predicted features to the acceptance region: minus
    the period's distance from the target in tolerances, plus half a ramp
    in log amplitude around AMP_MIN and half the oscillation indicator
    (both clipped to [0, 1]).  The GPU form is score_kernel in
    csrc/surrogate/features.cu."""
    per = np.exp(np.clip(log_per, -10.0, 10.0))
    amp_term = np.clip((log_amp - math.log(AMP_MIN)) / AMP_RAMP + 0.5, 0.0, 1.0)
    return -np.abs(per - TARGET_PERIOD) / PERIOD_TOL + 0.5 * amp_term + 0.5 * np.clip(p_osc, 0.0, 1.0)


def predicted_score(pred):
    """Higher is better: the predicted acceptance indicator plus
    REGION_WEIGHT times the predicted features' closeness to the acceptance
    region (the two together keep more of the candidates the FP64
    simulation accepts than either alone)."""
    pred = np.asarray(pred, np.float64)
    return pred[:, 4] + REGION_WEIGHT * _region_terms(pred[:, 0], pred[:, 1], pred[:, 3])


def score_candidates(net, P, chunk=1 << 20, spread=SPREAD, batch=65536):
    """predicted_score(net.predict(encode(P))) on the GPU: per chunk of
    candidates one host-to-device copy of their parameters, then the
    encoding, every network of the ensemble (`net` a Surrogate, or one MLP)
    and the score in the surrogate library's kernels; float64 numpy array."""
    import torch
    from .surrogate import IN_PAD
    nets = getattr(net, "nets", None) or [net]
    n_out = nets[0].n_out
    mu = getattr(net, "mu", np.zeros(n_out, np.float32))
    sd = getattr(net, "sd", np.ones(n_out, np.float32))
    dev = nets[0].dev
    k = nets[0].k
    idx = active_params()
    idx_d = torch.as_tensor(idx.astype(np.int32), device=dev)
    t_d = torch.as_tensor(template()[idx], device=dev, dtype=torch.float64)
    for m in nets:
        m._cast_weights()
    n = P.shape[0]
    out = torch.empty(n, dtype=torch.float64, device=dev)
    acc = torch.empty((batch, n_out), dtype=torch.float32, device=dev)
    for s in range(0, n, chunk):
        Pd = torch.as_tensor(np.ascontiguousarray(P[s:s + chunk], np.float64), device=dev)
        for b in range(0, Pd.shape[0], batch):
            rows = min(batch, Pd.shape[0] - b)
            Bp = (rows + 127) // 128 * 128
            Xb = nets[0]._buf("Xscore", (Bp, IN_PAD), torch.bfloat16)
            k.encode(Pd[b:b + rows], idx_d, t_d, math.log(spread), Xb)
            for i, m in enumerate(nets):
                k.ensemble_accumulate(m.forward(Xb), rows, n_out, acc, i == 0)
            k.score(acc[:rows], len(nets), mu, sd, REGION_WEIGHT, TARGET_PERIOD, PERIOD_TOL, AMP_MIN, AMP_RAMP,
                    out[s + b:s + b + rows])
    for m in nets:
        m.k.check()
    return out.cpu().numpy()


def feature_errors(net, P, F):
    """Relative error of predicted period and amplitude on sets that
    oscillate, against the FP64 simulation."""
    pred = net.predict(encode(P))
    osc = F["oscillates"] > 0.5
    per_err = np.abs(np.exp(pred[osc, 0]) - F["period"][osc]) / F["period"][osc]
    amp_err = np.abs(np.exp(pred[osc, 1]) - F["amplitude"][osc]) / F["amplitude"][osc]
    return {"period_median": float(np.median(per_err)), "amplitude_median": float(np.median(amp_err)),
            "period_p90": float(np.quantile(per_err, 0.9)), "amplitude_p90": float(np.quantile(amp_err, 0.9)),
            "oscillation_accuracy": float(((pred[:, 3] > 0.5) == osc).mean()), "n": int(osc.sum())}


def screened_search(net, n_candidates, seed, keep=0.01, plain_sample=4096, sim_kwargs=None, log=None):
    """Surrogate-screened search against plain GPU search on the same
    seeded candidates.  The surrogate ranks all candidates, its top `keep`
    fraction is simulated in FP64 and accepted by the simulation alone; the
    plain rate comes from simulating a random sample of the same candidates
    and is extrapolated per candidate."""
    sim_kwargs = sim_kwargs or {}
    P = draw_candidates(n_candidates, seed)
    from .distributed import local_top
    t0 = time.perf_counter()
    score = score_candidates(net, P)
    # the ranking counts the selection of the kept candidates too
    top = local_top(score, np.arange(n_candidates), max(1, int(round(keep * n_candidates))))[1]
    t_infer = time.perf_counter() - t0
    Fs = simulate_features(P[top], log=log, **sim_kwargs)
    acc_s = accepted(Fs)
    # surrogate error on the accepted sets, against their FP64 re-simulation
    pred_top = net.predict(encode(P[top]))
    with np.errstate(invalid="ignore", divide="ignore"):
        per_err = np.abs(np.exp(pred_top[acc_s, 0]) - Fs["period"][acc_s]) / Fs["period"][acc_s]
        amp_err = np.abs(np.exp(pred_top[acc_s, 1]) - Fs["amplitude"][acc_s]) / Fs["amplitude"][acc_s]
    t_screen = t_infer + Fs["seconds"]
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    sample = rng.choice(n_candidates, size=min(plain_sample, n_candidates), replace=False)
    Fp = simulate_features(P[sample], log=log, **sim_kwargs)
    acc_p = accepted(Fp)
    per_candidate = Fp["seconds"] / len(sample)
    plain_rate = acc_p.mean() / per_candidate if acc_p.any() else 0.0
    screened_rate = acc_s.sum() / t_screen
    return {
        "candidates": n_candidates, "kept": int(len(top)), "inference_s": t_infer,
        "resimulation_s": Fs["seconds"], "accepted_screened": int(acc_s.sum()),
        "false_accept_rate": float(1.0 - acc_s.mean()),
        "plain_sample": int(len(sample)), "plain_accept_fraction": float(acc_p.mean()),
        "plain_seconds_per_candidate": per_candidate,
        "accepted_per_s_screened": float(screened_rate), "accepted_per_s_plain": float(plain_rate),
        "gain": float(screened_rate / plain_rate) if plain_rate > 0 else float("inf"),
        "accepted_period_error_median": float(np.median(per_err)) if acc_s.any() else None,
        "accepted_amplitude_error_median": float(np.median(amp_err)) if acc_s.any() else None,
    }


def _draw_rows(rng, m, spread=SPREAD):
    t = template()
    return t[None, :] * np.exp(rng.uniform(np.log(1.0 / spread), np.log(spread), size=(m, t.size)))


def screened_search_sharded(net, n_candidates, seed, keep=0.01, group=None, sim_kwargs=None, log=None):
    """Surrogate-screened search over GPUs (one process per GPU): each rank
    draws and scores its contiguous share of the candidates (chunked seeded
    streams, dense_b200.distributed), the global top `keep` fraction is
    merged from the ranks' local tops, each rank re-simulates every
    world-th of it in FP64, and the accepted counts are summed.  Returns the
    totals (the same on every rank); times are the max over ranks."""
    import torch
    import torch.distributed as dist
    from . import distributed as D
    sim_kwargs = sim_kwargs or {}
    on = dist.is_available() and dist.is_initialized()
    rank = dist.get_rank(group) if on else 0
    world = dist.get_world_size(group) if on else 1
    lo, hi = D.shard_range(n_candidates, rank, world)
    t0 = time.perf_counter()
    P = D.candidate_range(lo, hi, seed, _draw_rows)
    score = score_candidates(net, P) if len(P) else np.zeros(0)
    top = D.global_top(score, np.arange(lo, hi), max(1, int(round(keep * n_candidates))), group)
    t_infer = time.perf_counter() - t0
    mine = top[rank::world]
    Fs = simulate_features(D.candidates_at(mine, seed, _draw_rows), log=log, **sim_kwargs) if len(mine) else None
    acc = int(accepted(Fs).sum()) if Fs is not None else 0
    sim_s = Fs["seconds"] if Fs is not None else 0.0
    vals = torch.tensor([float(acc), t_infer, sim_s], dtype=torch.float64)
    if on:
        if dist.get_backend(group) == "nccl":
            vals = vals.cuda()
        s = vals[:1].clone()
        dist.all_reduce(s, op=dist.ReduceOp.SUM, group=group)
        m = vals[1:].clone()
        dist.all_reduce(m, op=dist.ReduceOp.MAX, group=group)
        vals = torch.cat([s, m]).cpu()
    acc_total, t_inf, t_sim = float(vals[0]), float(vals[1]), float(vals[2])
    return {"candidates": n_candidates, "ranks": world, "kept": int(len(top)), "accepted_screened": int(acc_total),
            "inference_s": t_inf, "resimulation_s": t_sim,
            "accepted_per_s_screened": acc_total / max(1e-12, t_inf + t_sim)}


class SRES:
    """Stochastic-ranking evolution strategy (Runarsson & Yao, IEEE TEC 4(3),
    2000), the method of DENSE's search/ (libSRES), in the log-parameter box
    [-1, 1]^d of encode(): (mu, lambda) selection, self-adapted step sizes
    with exponential smoothing (alpha), differential variation for the
    parents (gamma).  The search is unconstrained, so stochastic ranking
    reduces to sorting by fitness.

    `fitness(X)` scores a whole population at once (one engine batch).
    With a surrogate, `screen` x lambda offspring are drawn and only the
    lambda the surrogate ranks best are scored by simulation.
    """

    def __init__(self, dim, fitness, mu=30, lam=200, seed=0, gamma=0.85, alpha=0.2, surrogate=None, screen=1):
        self.dim, self.fitness, self.mu, self.lam = dim, fitness, mu, lam
        self.gamma, self.alpha = gamma, alpha
        self.rng = np.random.Generator(np.random.PCG64(seed))
        self.tau = 1.0 / math.sqrt(2.0 * math.sqrt(dim))
        self.tau_p = 1.0 / math.sqrt(2.0 * dim)
        self.x = self.rng.uniform(-1, 1, size=(lam, dim))
        self.sigma = np.full((lam, dim), 2.0 / math.sqrt(dim))
        self.surrogate, self.screen = surrogate, max(1, screen)
        self.f = self.fitness(self.x)
        self.evaluations = lam

    def step(self):
        order = np.argsort(self.f, kind="stable")
        par_x, par_s = self.x[order[:self.mu]], self.sigma[order[:self.mu]]
        n_off = self.lam * self.screen
        pick = np.arange(n_off) % self.mu
        x, s = par_x[pick].copy(), par_s[pick].copy()
        # differential variation of the mu - 1 best (the SRES recombination)
        k = np.arange(n_off) < self.mu - 1
        x[k] = x[k] + self.gamma * (par_x[0] - par_x[(np.arange(n_off)[k] + 1) % self.mu])
        # self-adaptive mutation
        n0 = self.rng.normal(size=(n_off, 1))
        s_new = s * np.exp(self.tau_p * n0 + self.tau * self.rng.normal(size=s.shape))
        s_new = np.clip(s_new, 1e-4, 2.0)
        x_new = x + s_new * self.rng.normal(size=x.shape)
        x_new = np.where(np.abs(x_new) > 1.0, x - 0.5 * (x_new - x), x_new)
        x_new = np.clip(x_new, -1.0, 1.0)
        s = s + self.alpha * (s_new - s)
        if self.surrogate is not None and self.screen > 1:
            keep = np.argsort(-self.surrogate(x_new), kind="stable")[:self.lam]
            x_new, s = x_new[keep], s[keep]
        self.x, self.sigma = x_new, s
        self.f = self.fitness(self.x)
        self.evaluations += len(self.x)
        return float(np.min(self.f))


def decode(X, spread=SPREAD):
    """Inverse of encode: [n][d] in [-1, 1] -> full parameter rows."""
    t = template()
    P = np.tile(t, (X.shape[0], 1))
    P[:, active_params()] = t[active_params()] * np.exp(X * math.log(spread))
    return P


def search_fitness(F):
    """Lower is better: distance of the period to the target window, plus a
    penalty below the amplitude threshold; sets that do not oscillate score 1e3."""
    per, amp = F["period"], np.nan_to_num(F["amplitude"])
    with np.errstate(invalid="ignore"):
        f = np.abs(per - TARGET_PERIOD) / PERIOD_TOL + np.maximum(0.0, AMP_MIN - amp) / AMP_MIN
    return np.where(np.isfinite(f), f, 1e3)
