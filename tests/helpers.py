"""Runs a golden case through the engine, the oracle, or reads DENSE's fixture."""

import math
import os

import numpy as np

from tests.golden.cases import build_case

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_fixture(name):
    return dict(np.load(os.path.join(GOLDEN, "ref_%s.npz" % name)))


def run_oracle(lib, name):
    """Same outputs as make_goldens.run_ref, from an oracle library."""
    case = build_case(name)
    out = {}
    for s, ps in enumerate(case["sets"]):
        sim = lib.create(ps["off"], ps["ids"], ps["cell_params"], ps["set_params"], ps["init_conc"], case["dt"],
                         ps.get("perturb"))
        for a in case["analyses"]:
            if a["kind"] == "basic":
                sim.add_basic(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1])
            elif a["kind"] == "oscillation":
                sim.add_oscillation(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"],
                                    a["intvl"])
            else:
                sim.add_conccheck(a["target"], a["cells"][0], a["cells"][1], a["lo"], a["hi"], a["t"][0], a["t"][1])
        out["chunks_%d" % s] = sim.run(ps["duration"], case["interval"])
        out["status_%d" % s] = np.int32(sim.status())
        out["state_%d" % s] = sim.state()
        out["S_%d" % s] = sim.ring_sizes()[0]
        for i, a in enumerate(case["analyses"]):
            if a["kind"] == "basic":
                b = sim.basic(i)
                for k in ("mins", "sums", "maxs", "samples", "time"):
                    out["a%d_%s_%d" % (i, k, s)] = np.asarray(b[k])
                if a["cells"][0] == 0:
                    for k in ("cell_mins", "cell_sums", "cell_maxs"):
                        out["a%d_%s_%d" % (i, k, s)] = b[k]
            elif a["kind"] == "oscillation":
                o = sim.oscillation(i)
                for k in ("amps", "pers", "avg_peak", "ncrit", "samples", "time"):
                    out["a%d_%s_%d" % (i, k, s)] = np.asarray(o[k])
    return out


def run_engine(name, precision=0, graph=False, chunks_per_call=-1, schedule=0):
    """The case through the CUDA engine (one batch holding all its sets,
    every set with the schedule hint `schedule`)."""
    from dense_b200.engine import Analysis, Batch, ParameterSet
    case = build_case(name)
    sets = [ParameterSet(ps["off"], ps["ids"], ps["set_params"], cell_params=ps["cell_params"],
                         init_conc=ps["init_conc"], perturb=ps.get("perturb"), duration=ps["duration"],
                         schedule=schedule)
            for ps in case["sets"]]
    an = []
    for a in case["analyses"]:
        if a["kind"] == "basic":
            an.append(Analysis.basic(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1]))
        elif a["kind"] == "oscillation":
            an.append(Analysis.oscillation(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1],
                                           a["win"], a["intvl"]))
        else:
            # DENSE's check takes one target species, or every species (-1)
            an.append(Analysis.conccheck([a["target"]] if a["target"] >= 0 else [], a["cells"][0], a["cells"][1],
                                         a["lo"], a["hi"], a["t"][0], a["t"][1]))
    b = Batch(case["model"], sets, case["dt"], case["interval"], an, precision=precision)
    if chunks_per_call < 0:
        b.run(-1, graph=graph)
    else:
        total = max(int(math.ceil(ps["duration"] / case["interval"])) for ps in case["sets"])
        for _ in range(0, total + chunks_per_call, chunks_per_call):
            b.run(chunks_per_call, graph=graph)
    b.sync()
    out = {}
    status = b.status()
    chunks, _ = b.progress()
    for s in range(len(sets)):
        out["status_%d" % s] = status[s]
        out["chunks_%d" % s] = chunks[s]
        out["state_%d" % s] = b.state(s)
        out["S_%d" % s] = b.ring_info(s)[0]
        for i, a in enumerate(case["analyses"]):
            if a["kind"] == "basic":
                r = b.basic(i, s)
                for k in ("mins", "sums", "maxs", "samples", "time"):
                    out["a%d_%s_%d" % (i, k, s)] = np.asarray(r[k])
                if a["cells"][0] == 0:
                    for k in ("cell_mins", "cell_sums", "cell_maxs"):
                        out["a%d_%s_%d" % (i, k, s)] = r[k]
            elif a["kind"] == "oscillation":
                r = b.oscillation(i, s)
                for k in ("amps", "pers", "avg_peak", "ncrit", "samples", "time"):
                    out["a%d_%s_%d" % (i, k, s)] = np.asarray(r[k])
    b.close()
    return out


def same(a, b):
    """Bitwise equality with every NaN equal to every NaN."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f" or b.dtype.kind == "f":
        a = a.astype(np.float64)
        b = b.astype(np.float64)
        na, nb = np.isnan(a), np.isnan(b)
        return bool(np.array_equal(na, nb) and np.array_equal(a[~na], b[~nb]))
    return bool(np.array_equal(a, b))


def mismatches(expected, got, keys=None):
    bad = []
    for k in (keys or expected):
        if k not in got:
            bad.append((k, "missing"))
        elif not same(expected[k], got[k]):
            e = np.asarray(expected[k], np.float64)
            g = np.asarray(got[k], np.float64)
            with np.errstate(invalid="ignore", divide="ignore"):
                rel = np.nanmax(np.abs(e - g) / np.maximum(np.abs(e), 1e-300)) if e.shape == g.shape else None
            bad.append((k, rel))
    return bad
