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
