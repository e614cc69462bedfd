"""The small parity cases shared by the golden-fixture script and the tests.

Every input is generated from a seed (numpy PCG64) and the model templates
in dense_b200/data/templates.json, so the engine, the oracle and DENSE
itself see identical inputs.
"""

import numpy as np

from dense_b200 import workloads
from dense_b200.tissue import default_graph

INF = float("inf")


def _her(*names):
    return workloads.her_species(*names)


def _set(model, cells, width, duration, cell_params=None, set_params=None, init_conc=None, perturb=None):
    off, ids = default_graph(cells, width)
    p = workloads.template_params(model) if set_params is None else np.asarray(set_params, np.float64)
    cp = np.tile(p, (cells, 1)) if cell_params is None else cell_params
    return dict(off=off, ids=ids, set_params=p, cell_params=cp, init_conc=init_conc, perturb=perturb,
                duration=duration)


def _her_test():
    # DENSE's CTest "her_test" (test/her_model_2014/CMakeLists.txt:9-18,
    # analyses.xml) minus its second Basic analysis, whose cell range
    # (0-19) lies outside the 10-cell tissue.
    return dict(model="her_model_2014", dt=0.01, interval=0.01,
                sets=[_set("her_model_2014", 10, 5, 3000.0)],
                analyses=[dict(kind="basic", species=_her("ph1", "ph7"), cells=(0, 9), t=(0.0, 15.0)),
                          dict(kind="oscillation", species=_her("ph1", "mh1", "md"), cells=(0, 5), t=(0.0, 60.0),
                               win=4.0, intvl=0.01)])


def _her_pert():
    ps = workloads.perturbed_set(cells=200, width=4, duration=60.0, seed=1)
    nsp = len(workloads.templates()["her_model_2014"]["species"])
    return dict(model="her_model_2014", dt=0.01, interval=0.1,
                sets=[_set("her_model_2014", 200, 4, 60.0, cell_params=ps.cell_params)],
                analyses=[dict(kind="basic", species=list(range(nsp)), cells=(0, 200), t=(0.0, INF)),
                          dict(kind="oscillation", species=_her("mh1", "ph1"), cells=(0, 200), t=(0.0, INF),
                               win=4.0, intvl=0.1)])


def _her_sets():
    P = workloads.log_uniform_params(6, 0.5, 2.0, seed=3)
    return dict(model="her_model_2014", dt=0.01, interval=0.1,
                sets=[_set("her_model_2014", 32, 4, 120.0, set_params=P[i]) for i in range(6)],
                analyses=[dict(kind="basic", species=_her("mh1", "pd"), cells=(0, 32), t=(0.0, INF)),
                          dict(kind="oscillation", species=_her("mh1"), cells=(0, 32), t=(0.0, INF), win=4.0,
                               intvl=0.1)])


def _her_delays():
    # delays drawn from [5, 20] minutes per set, per-cell +-5% on top
    base = workloads.template_params()
    rng = np.random.Generator(np.random.PCG64(4))
    sets = []
    for i in range(4):
        p = base.copy()
        p[34:42] = np.where(p[34:42] > 0, rng.uniform(5.0, 20.0, 8), 0.0)
        cp = p[None, :] * rng.uniform(0.95, 1.05, size=(16, p.size))
        sets.append(_set("her_model_2014", 16, 4, 60.0, cell_params=cp, set_params=p))
    return dict(model="her_model_2014", dt=0.01, interval=0.1, sets=sets,
                analyses=[dict(kind="oscillation", species=_her("mh1", "md"), cells=(0, 16), t=(0.0, INF),
                               win=2.0, intvl=0.1)])


def _her_init():
    ic = workloads.templates()["her_model_2014"]["init_conc"]
    nsp = len(ic)
    return dict(model="her_model_2014", dt=0.01, interval=0.05,
                sets=[_set("her_model_2014", 20, 5, 30.0, init_conc=np.array(ic))],
                analyses=[dict(kind="basic", species=list(range(nsp)), cells=(0, 20), t=(0.0, INF))])


def _turing():
    ic = workloads.templates()["turing"]["init_conc"]
    return dict(model="turing", dt=0.01, interval=0.5,
                sets=[_set("turing", 64, 8, 10.0, init_conc=np.array(ic))],
                analyses=[dict(kind="basic", species=[0, 1, 2, 3], cells=(0, 64), t=(0.0, INF))])


def _nan_test():
    # DENSE's CTest "nan_test" (test/Nan_Test/CMakeLists.txt:6-16).
    return dict(model="nan_test", dt=0.01, interval=0.5,
                sets=[_set("nan_test", 100, 100, 15.0)],
                analyses=[dict(kind="basic", species=[0, 1, 2], cells=(0, 99), t=(0.0, 2.0))])


def _other(model, seed, delay_sets=()):
    # DENSE's other example models (their templates hold zero rates):
    # seeded positive rates U[0.05, 2), initial concentrations U[0, 5),
    # 24 cells of width 6, 4 minutes; one set with delays U[0.5, 4) and one
    # per entry of `delay_sets` (explicit delays, e.g. the template's
    # 100-minute ones, whose reads only ever see the initial rows)
    rng = np.random.Generator(np.random.PCG64(seed))
    t = workloads.templates()[model]
    nsp, nr = len(t["species"]), len(t["reactions"])
    p = rng.uniform(0.05, 2.0, size=t["num_params"])
    nd = t["num_params"] - nr if model == "delay_reaction" else 0
    p[nr:nr + nd] = rng.uniform(0.5, 4.0, nd)
    ic = rng.uniform(0.0, 5.0, size=nsp)
    sets = [_set(model, 24, 6, 4.0, set_params=p, init_conc=ic)]
    for d in delay_sets:
        q = p.copy()
        q[nr:nr + nd] = d
        sets.append(_set(model, 24, 6, 4.0, set_params=q, init_conc=ic))
    return dict(model=model, dt=0.01, interval=0.1, sets=sets,
                analyses=[dict(kind="basic", species=list(range(nsp)), cells=(0, 24), t=(0.0, INF)),
                          dict(kind="oscillation", species=[0], cells=(0, 24), t=(0.0, INF), win=1.0, intvl=0.1)])


def _her_pert_factors():
    # -b perturbation factors per reaction: they scale the delays that size
    # DENSE's rings (base.cpp:55-140), so reads at lag S-1 (delays below one
    # minute truncate to k = 0) see other rows
    rng = np.random.Generator(np.random.PCG64(5))
    nsp = len(workloads.templates()["her_model_2014"]["species"])
    return dict(model="her_model_2014", dt=0.01, interval=0.1,
                sets=[_set("her_model_2014", 20, 4, 30.0, perturb=rng.uniform(0.0, 0.6, size=34))],
                analyses=[dict(kind="basic", species=list(range(nsp)), cells=(0, 20), t=(0.0, INF)),
                          dict(kind="oscillation", species=_her("mh1", "mh13"), cells=(0, 20), t=(0.0, INF),
                               win=4.0, intvl=0.1)])


def _her_conccheck():
    # ConcentrationCheck (conccheck.hpp:25-51) with run_simulation's drop
    # (run_simulation.hpp:131-150): a check of mh1 over every cell in [0,
    # 150] during the first 15 minutes drops four of the eight sets at
    # different chunks, a check of every species of cells 4-11 in [-1,
    # 20000] during minutes 20-50 drops two more, two sets run to the end
    P = workloads.log_uniform_params(8, seed=41)
    return dict(model="her_model_2014", dt=0.01, interval=0.1,
                sets=[_set("her_model_2014", 16, 4, 60.0, set_params=P[i]) for i in range(8)],
                analyses=[dict(kind="basic", species=_her("mh1", "pd"), cells=(0, 16), t=(0.0, INF)),
                          dict(kind="conccheck", target=_her("mh1")[0], cells=(0, 16), lo=0.0, hi=150.0,
                               t=(0.0, 15.0)),
                          dict(kind="conccheck", target=-1, cells=(4, 12), lo=-1.0, hi=20000.0, t=(20.0, 50.0))])


CASES = {
    "her_test": _her_test,
    "her_pert": _her_pert,
    "her_sets": _her_sets,
    "her_delays": _her_delays,
    "her_init": _her_init,
    "her_pert_factors": _her_pert_factors,
    "her_conccheck": _her_conccheck,
    "turing": _turing,
    "nan_test": _nan_test,
    "delay_reaction": lambda: _other("delay_reaction", 21, delay_sets=[(100.0, 100.0)]),
    "bz": lambda: _other("bz", 22),
    "briggs_rauscher": lambda: _other("briggs_rauscher", 23),
}


# ---- the configurations at their full sizes (one set, the batched
# workload's own sets, the largest shapes of the uneven mixed batch): DENSE
# itself makes the fixtures; the engine's GPU tests compare with them bit
# for bit.  Kept out of CASES, whose cases the CPU tests also run through
# the oracle in seconds.

CFG2_SETS = 4096      # the batched workload: log_uniform_sets(4096, seed=2), 200 cells, 1200 min
CFG2_PICK = 4         # sets taken from each end of the truncated-delay ranking


def cfg2_indices():
    """The batched workload's sets with the fewest and the most minutes of
    truncated delay (the sum over delay reactions of int(delay), the lag
    DENSE reads at): CFG2_PICK of each, in index order."""
    P = workloads.log_uniform_params(CFG2_SETS, seed=2)
    nr = len(workloads.templates()["her_model_2014"]["reactions"])
    k = np.floor(P[:, nr:nr + 8]).sum(axis=1)
    order = np.argsort(k, kind="stable")
    return sorted(int(i) for i in np.concatenate([order[:CFG2_PICK], order[-CFG2_PICK:]]))


def _her_cfg1_full():
    # the one-set configuration: 200 cells, every parameter of every cell
    # x U(0.95, 1.05), 600 min, Basic over every species and cell +
    # Oscillation of mh1 and ph1 every 0.1 min
    ps = workloads.perturbed_set(cells=200, width=4, duration=600.0, seed=1)
    nsp = len(workloads.templates()["her_model_2014"]["species"])
    return dict(model="her_model_2014", dt=0.01, interval=0.1,
                sets=[_set("her_model_2014", 200, 4, 600.0, cell_params=ps.cell_params)],
                analyses=[dict(kind="basic", species=list(range(nsp)), cells=(0, 200), t=(0.0, INF)),
                          dict(kind="oscillation", species=_her("mh1", "ph1"), cells=(0, 200), t=(0.0, INF),
                               win=4.0, intvl=0.1)])


def _her_cfg2_full():
    # the batched configuration's own sets (see cfg2_indices), 200 cells,
    # 1200 min, Oscillation of mh1 over every cell every 0.1 min
    P = workloads.log_uniform_params(CFG2_SETS, seed=2)
    idx = cfg2_indices()
    return dict(model="her_model_2014", dt=0.01, interval=0.1, indices=idx,
                sets=[_set("her_model_2014", 200, 4, 1200.0, set_params=P[i]) for i in idx],
                analyses=[dict(kind="oscillation", species=_her("mh1"), cells=(0, 200), t=(0.0, INF), win=4.0,
                               intvl=0.1)])


def _her_cfg3_large():
    # the mixed batch's largest her_model_2014 shape: 1024 cells (-w 4),
    # every rate x exp(U(ln 1/2, ln 2)), every delay U[5, 20] min, 1200 min
    rng = np.random.Generator(np.random.PCG64(31))
    p = workloads.template_params()
    p = p * np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=p.size))
    nr = len(workloads.templates()["her_model_2014"]["reactions"])
    p[nr:nr + 8] = rng.uniform(5.0, 20.0, size=8)
    nsp = len(workloads.templates()["her_model_2014"]["species"])
    return dict(model="her_model_2014", dt=0.01, interval=0.1,
                sets=[_set("her_model_2014", 1024, 4, 1200.0, set_params=p)],
                analyses=[dict(kind="basic", species=list(range(nsp)), cells=(0, 1024), t=(0.0, INF)),
                          dict(kind="oscillation", species=_her("mh1"), cells=(0, 1024), t=(0.0, INF), win=4.0,
                               intvl=0.1)])


def _her_cfg3_large_cells():
    # the same set with every parameter of every cell x U(0.95, 1.05) on
    # top, so the 1024 cells differ and every neighbour read matters
    case = _her_cfg3_large()
    p = case["sets"][0]["set_params"]
    rng = np.random.Generator(np.random.PCG64(33))
    cp = p[None, :] * rng.uniform(0.95, 1.05, size=(1024, p.size))
    case["sets"] = [_set("her_model_2014", 1024, 4, 1200.0, cell_params=cp, set_params=p)]
    return case


def _turing_cfg3_large():
    # the mixed batch's largest Turing-Pattern shape: a 64 x 64 grid
    # (-c 4096 -w 64), every parameter x exp(U(ln 1/2, ln 2)), the model's
    # initial concentrations, 1200 min
    rng = np.random.Generator(np.random.PCG64(32))
    p = workloads.template_params("turing")
    p = p * np.exp(rng.uniform(np.log(0.5), np.log(2.0), size=p.size))
    ic = workloads.templates()["turing"]["init_conc"]
    return dict(model="turing", dt=0.01, interval=1.0,
                sets=[_set("turing", 4096, 64, 1200.0, set_params=p, init_conc=np.array(ic))],
                analyses=[dict(kind="basic", species=[0, 1, 2, 3], cells=(0, 4096), t=(0.0, INF))])


FULL_CASES = {
    "her_cfg1_full": _her_cfg1_full,
    "her_cfg2_full": _her_cfg2_full,
    "her_cfg3_large": _her_cfg3_large,
    "her_cfg3_large_cells": _her_cfg3_large_cells,
    "turing_cfg3_large": _turing_cfg3_large,
}


def build_case(name):
    return CASES[name]() if name in CASES else FULL_CASES[name]()
