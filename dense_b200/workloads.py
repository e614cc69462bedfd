"""Seeded synthetic workloads of the her_model_2014 benchmark configurations.

No dataset is involved: every input is generated from the model's template
parameter set (data/templates.json, the first set of the model's
param_sets.csv) with numpy's PCG64 generator.

* ``tissue_200``: DENSE's default hexagonal tissue, 200 cells, width 4
  (``-c 200 -w 4``).
* ``perturbed_set``: one set, every parameter of every cell multiplied by
  U(0.95, 1.05) -- an explicit per-cell matrix (DENSE's own ``-b`` path
  reads past the end of its factor array, sim/base.cpp:13-15).
* ``log_uniform_sets``: each set scales every template parameter by
  exp(U(ln lo, ln hi)); zero parameters stay zero.
"""

import json
import os

import numpy as np

from .engine import Analysis, ParameterSet
from .tissue import default_graph

HERE = os.path.dirname(os.path.abspath(__file__))


def templates():
    with open(os.path.join(HERE, "data", "templates.json")) as f:
        return json.load(f)


def template_params(model="her_model_2014"):
    return np.array(templates()[model]["params"], np.float64)


def perturbed_set(model="her_model_2014", cells=200, width=4, duration=600.0, spread=0.05, seed=1,
                  init_conc=None):
    p = template_params(model)
    rng = np.random.Generator(np.random.PCG64(seed))
    cell = p[None, :] * rng.uniform(1.0 - spread, 1.0 + spread, size=(cells, p.size))
    off, ids = default_graph(cells, width)
    return ParameterSet(off, ids, p, cell_params=cell, init_conc=init_conc, duration=duration)


def log_uniform_params(num_sets, lo=0.5, hi=2.0, seed=2, model="her_model_2014"):
    p = template_params(model)
    rng = np.random.Generator(np.random.PCG64(seed))
    f = np.exp(rng.uniform(np.log(lo), np.log(hi), size=(num_sets, p.size)))
    return p[None, :] * f


def log_uniform_sets(num_sets, cells=200, width=4, duration=1200.0, lo=0.5, hi=2.0, seed=2,
                     model="her_model_2014"):
    P = log_uniform_params(num_sets, lo, hi, seed, model)
    off, ids = default_graph(cells, width)
    return [ParameterSet(off, ids, P[i], duration=duration) for i in range(num_sets)]


def her_species(*names):
    sp = templates()["her_model_2014"]["species"]
    return [sp.index(n) for n in names]


def cfg1_analyses(cells=200, interval=0.1):
    """Basic over every species and cell, Oscillation of mh1 and ph1
    (4-minute window, sampled every `interval`)."""
    nsp = len(templates()["her_model_2014"]["species"])
    return [Analysis.basic(list(range(nsp)), 0, cells),
            Analysis.oscillation(her_species("mh1", "ph1"), 0, cells, 0.0, float("inf"), 4.0, interval)]


def batch_analyses(cells=200, interval=0.1):
    """Per-set oscillation period and amplitude of mh1 over every cell."""
    return [Analysis.oscillation(her_species("mh1"), 0, cells, 0.0, float("inf"), 4.0, interval)]


def mixed_sets(num_sets, seed=3, her_fraction=0.5, lo=0.5, hi=2.0):
    """The uneven mixed batch: `num_sets` sets split between her_model_2014
    and Turing-Pattern (each set her with probability `her_fraction`).

    * her_model_2014: cell count log-uniform over [16, 1024] in multiples of
      4 on DENSE's default tissue of width 4 (``-c n -w 4``); every rate
      scaled by exp(U(ln lo, ln hi)); every delay U[5, 20] min.
    * Turing-Pattern: an N x N grid, N uniform in [8, 64] (``-c N*N -w N``);
      every parameter scaled by exp(U(ln lo, ln hi)); the model's initial
      concentrations.
    * horizons U[100, 1200] min for both.

    Returns {"her_model_2014": [ParameterSet], "turing": [ParameterSet]}.
    """
    from .engine import load
    rng = np.random.Generator(np.random.PCG64(seed))
    hp, tp = template_params("her_model_2014"), template_params("turing")
    L = load("her_model_2014")
    d0, d1 = L.num_reactions, L.num_reactions + L.num_delay_reactions
    tinit = np.array(templates()["turing"]["init_conc"], np.float64)
    graphs = {}

    def graph(n, w):
        if (n, w) not in graphs:
            graphs[(n, w)] = default_graph(n, w)
        return graphs[(n, w)]

    out = {"her_model_2014": [], "turing": []}
    for _ in range(num_sets):
        horizon = float(rng.uniform(100.0, 1200.0))
        if rng.random() < her_fraction:
            n = 4 * int(round(np.exp(rng.uniform(np.log(4), np.log(256)))))
            p = hp * np.exp(rng.uniform(np.log(lo), np.log(hi), size=hp.size))
            p[d0:d1] = rng.uniform(5.0, 20.0, size=d1 - d0)
            off, ids = graph(n, 4)
            out["her_model_2014"].append(ParameterSet(off, ids, p, duration=horizon))
        else:
            N = int(rng.integers(8, 65))
            p = tp * np.exp(rng.uniform(np.log(lo), np.log(hi), size=tp.size))
            off, ids = graph(N * N, N)
            out["turing"].append(ParameterSet(off, ids, p, init_conc=tinit, duration=horizon))
    return out
