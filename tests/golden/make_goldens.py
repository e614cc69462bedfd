"""Generates the golden fixtures under tests/golden/.

1. ``dense_ctest/``: the blessed output files of DENSE's own CTest suite for
   the deterministic path, copied verbatim as data
   (test/her_model_2014/{anlys_basic_a,anlys_oscil,cell_width_test_anlys,
   total_time_test_anlys,total_time_test_01_anlys}.csv and
   test/Nan_Test/anlys_basic_a.csv).
2. ``inputs/`` and ``cli/<case>/``: DENSE's own ``simulation`` command
   (oracle/_ref/<model>_simulation) run on CLI_CASES, its input files and
   the output files it wrote.
3. ``ref_<case>.npz``: full-precision outputs of DENSE itself (compiled from
   its sources into oracle/_ref/ by oracle/build.py and driven through
   oracle/ref_harness.cpp) on the small cases of CASES and, named on the
   command line, the full-size configurations of FULL_CASES (cases.py).
   The GPU tests compare the engine with these on machines without the
   DENSE tree.

Usage: python tests/golden/make_goldens.py [case ...]   (needs the DENSE tree)
"""

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.build import use_default_tree  # noqa: E402

use_default_tree()

from dense_b200.models import dense_dir  # noqa: E402
from tests.golden.cases import CASES, build_case  # noqa: E402

CTEST = {
    "her_anlys_basic_a.csv": "test/her_model_2014/anlys_basic_a.csv",
    "her_anlys_oscil.csv": "test/her_model_2014/anlys_oscil.csv",
    "her_cell_width_test_anlys.csv": "test/her_model_2014/cell_width_test_anlys.csv",
    "her_total_time_test_anlys.csv": "test/her_model_2014/total_time_test_anlys.csv",
    "her_total_time_test_01_anlys.csv": "test/her_model_2014/total_time_test_01_anlys.csv",
    "nan_anlys_basic_a.csv": "test/Nan_Test/anlys_basic_a.csv",
}


# Input files of the command-line cases, copied as data.
INPUTS = {
    "her_param_sets.csv": "test/her_model_2014/param_sets.csv",
    "her_analyses.xml": "test/her_model_2014/analyses.xml",
    "nan_param_sets.csv": "test/Nan_Test/param_sets.csv",
    "nan_analyses.xml": "test/Nan_Test/analyses.xml",
    "turing_param_sets.csv": "models/Turing-Pattern/param_sets.csv",
    "turing_init_conc.csv": "models/Turing-Pattern/init_conc.csv",
    "organic2.graphml": "models/Turing-Pattern/organic2.graphml",
    "cell_adj.g": "models/Turing-Pattern/cell_adj.g",
}

# DENSE's own `simulation` command (oracle/_ref/<model>_simulation) on these
# arguments writes the expected files; {in} is the inputs directory.
CLI_CASES = {
    "her_test": ("her_model_2014",
                 "-p {in}/her_param_sets.csv --cell-total 10 --tissue-width 5 --time-total 3000 --anlys-intvl .01 "
                 "--step-size .01 --analysis {in}/her_analyses.xml", ["anlys_basic_a.csv", "anlys_oscil.csv"]),
    # the other her_model_2014 CTest runs (test/her_model_2014/CMakeLists.txt:20-90):
    # tissue width, cell count and total time; with 20 or more cells the
    # second Basic (cells 0-19) lies in the tissue and is compared too
    "her_cell_width_test": ("her_model_2014",
                            "--param-sets {in}/her_param_sets.csv --cell-total 10 --tissue-width 1 --time-total 3000 "
                            "--anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                            ["anlys_basic_a.csv", "anlys_oscil.csv"]),
    "her_cell_width_test_01": ("her_model_2014",
                               "--param-sets {in}/her_param_sets.csv --cell-total 50 --tissue-width 10 "
                               "--time-total 3000 --anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                               ["anlys_basic_a.csv", "anlys_basic_b.csv", "anlys_oscil.csv"]),
    "her_cell_width_test_02": ("her_model_2014",
                               "--param-sets {in}/her_param_sets.csv --cell-total 100 --tissue-width 10 "
                               "--time-total 3000 --anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                               ["anlys_basic_a.csv", "anlys_basic_b.csv", "anlys_oscil.csv"]),
    "her_cell_number_test": ("her_model_2014",
                             "--param-sets {in}/her_param_sets.csv --cell-total 50 --tissue-width 5 "
                             "--time-total 3000 --anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                             ["anlys_basic_a.csv", "anlys_basic_b.csv", "anlys_oscil.csv"]),
    "her_cell_number_test_01": ("her_model_2014",
                                "--param-sets {in}/her_param_sets.csv --cell-total 200 --tissue-width 5 "
                                "--time-total 3000 --anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                                ["anlys_basic_a.csv", "anlys_basic_b.csv", "anlys_oscil.csv"]),
    "her_time_total_test": ("her_model_2014",
                            "--param-sets {in}/her_param_sets.csv --cell-total 10 --tissue-width 5 --time-total 300 "
                            "--anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                            ["anlys_basic_a.csv", "anlys_oscil.csv"]),
    "her_time_total_test_01": ("her_model_2014",
                               "--param-sets {in}/her_param_sets.csv --cell-total 10 --tissue-width 5 "
                               "--time-total 5000 --anlys-intvl .01 --step-size .01 --analysis {in}/her_analyses.xml",
                               ["anlys_basic_a.csv", "anlys_oscil.csv"]),
    "nan_test": ("nan_test",
                 "--param-sets {in}/nan_param_sets.csv --cell-total 100 --tissue-width 100 --time-total 15 "
                 "--anlys-intvl 0.5 -s 0.01 --analysis {in}/nan_analyses.xml", ["anlys_basic_a.csv"]),
    "turing_graphml_export": ("turing",
                              "-p {in}/turing_param_sets.csv -f {in}/organic2.graphml -t 4 -u 0.5 -s 0.01 "
                              "-d {in}/turing_init_conc.csv -e traj.csv -v", ["traj.csv"]),
    # a trajectory export with its time column and species in non-id order:
    # also the input of the -i (imported trajectory) cases below
    "her_traj_export_v": ("her_model_2014",
                          "-p {in}/her_param_sets.csv -c 12 -w 4 -t 30 -u 0.1 -s 0.01 -e traj.csv -v 1 "
                          "-o \"ph1, mh1, md\"", ["traj.csv"]),
    "her_edge_list_export": ("her_model_2014",
                             "-p {in}/her_param_sets.csv -f {in}/cell_adj.g -t 30 -u 1 -s 0.01 -e traj.csv "
                             "-o \"mh1, ph1\"", ["traj.csv"]),
}


def copy_inputs():
    out = os.path.join(HERE, "inputs")
    os.makedirs(out, exist_ok=True)
    for dst, src in INPUTS.items():
        shutil.copyfile(os.path.join(dense_dir(), src), os.path.join(out, dst))


def run_cli_cases():
    import shlex
    import subprocess
    import tempfile
    from oracle.build import build_ref, ref_cli_path
    inputs = os.path.join(HERE, "inputs")
    for name, (model, args, outs) in CLI_CASES.items():
        build_ref(model)
        exe = ref_cli_path(model)
        dst = os.path.join(HERE, "cli", name)
        os.makedirs(dst, exist_ok=True)
        with tempfile.TemporaryDirectory() as tmp:
            cmd = [exe] + shlex.split(args.format(**{"in": inputs}))
            r = subprocess.run(cmd, cwd=tmp, stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            # DENSE aborts at exit ("free(): invalid pointer") after a run on
            # an edge-list tissue; its output files are complete by then
            if r.returncode != 0 and not all(os.path.exists(os.path.join(tmp, f)) for f in outs):
                raise RuntimeError("DENSE failed on %s" % name)
            for f in outs:
                shutil.copyfile(os.path.join(tmp, f), os.path.join(dst, f))
                if f in UNDEFINED_ROWS:
                    _blank_undefined_rows(os.path.join(dst, f), UNDEFINED_ROWS[f])
        print("cli", name, outs)


# Rows DENSE prints from past the end of its per-species vectors
# (BasicAnalysis::show indexes them by species id, measurement/basic.ipp:
# 69-72; in anlys_basic_b the ids of mh1 and mh13 exceed its three observed
# species): their numbers change from run to run, so the fixture keeps the
# species name and marks the values undefined.
UNDEFINED_ROWS = {"anlys_basic_b.csv": ("mh1,", "mh13,")}


def _blank_undefined_rows(path, prefixes):
    with open(path) as f:
        lines = f.read().split("\n")
    lines = [ln.split(",")[0] + ",undefined,undefined,undefined" if ln.startswith(prefixes) else ln
             for ln in lines]
    with open(path, "w") as f:
        f.write("\n".join(lines))


def copy_ctest():
    out = os.path.join(HERE, "dense_ctest")
    os.makedirs(out, exist_ok=True)
    for dst, src in CTEST.items():
        shutil.copyfile(os.path.join(dense_dir(), src), os.path.join(out, dst))


def _ref_set(args):
    """DENSE's outputs for set `s` of case `name` (keys as in the fixtures)."""
    name, s = args
    from oracle.pyoracle import load_ref
    case = build_case(name)
    R = load_ref(case["model"])
    if R is None:
        raise RuntimeError("DENSE harness not built")
    ps = case["sets"][s]
    out = {}
    sim = R.create(ps["off"], ps["ids"], ps["cell_params"], ps["set_params"], ps["init_conc"], case["dt"],
                   ps.get("perturb"))
    for a in case["analyses"]:
        if a["kind"] == "basic":
            sim.add_basic(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1])
        elif a["kind"] == "oscillation":
            sim.add_oscillation(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"],
                                a["intvl"])
        elif a["kind"] == "conccheck":
            if sim.add_conccheck(a["target"], a["cells"][0], a["cells"][1], a["lo"], a["hi"], a["t"][0],
                                 a["t"][1]) < 0:
                raise RuntimeError("DENSE harness without a concentration check")
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


def run_ref(name):
    """DENSE on every set of the case (sets in parallel host processes,
    each DENSE single-threaded as it is)."""
    import multiprocessing as mp
    case = build_case(name)
    n = len(case["sets"])
    jobs = [(name, s) for s in range(n)]
    if n > 1:
        with mp.get_context("spawn").Pool(min(n, os.cpu_count() or 1)) as pool:
            parts = pool.map(_ref_set, jobs)
    else:
        parts = [_ref_set(jobs[0])]
    out = {}
    for part in parts:
        out.update(part)
    if "indices" in case:
        out["indices"] = np.asarray(case["indices"], np.int64)
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **out)
    print("ref_%s.npz" % name, len(out), "arrays")


# Analysis of imported trajectories (simulation -i): the trajectory file,
# its analyses (analyses.xml text for the command, dicts for the harness),
# -t and -u.  Fixture ref_<name>.npz: DENSE's own BasicAnalysis and
# OscillationAnalysis over the file's samples (oracle_replay of the harness).
IMPORT_CASES = {
    "her_import_dense_export": dict(
        file="cli/her_traj_export_v/traj.csv", minutes=30.0, interval=0.1,
        analyses=[dict(kind="basic", species=["ph1", "mh1", "md"], cells=(0, 12), t=(0.0, 1e9)),
                  dict(kind="oscillation", species=["mh1", "ph1"], cells=(0, 12), t=(0.0, 1e9), win=2.0, intvl=0.1)]),
    "her_import_waves": dict(
        file="inputs/her_traj_waves.csv", minutes=20.0, interval=0.1,
        analyses=[dict(kind="basic", species=["mh1", "pd"], cells=(0, 7), t=(6.0, 1e9)),
                  dict(kind="oscillation", species=["mh1"], cells=(0, 7), t=(5.0, 1e9), win=3.0, intvl=0.1)]),
}


def write_waves_trajectory():
    """A seeded synthetic trajectory export (no DENSE run behind it): 10
    cells of which 0-6 are exported, pd and mh1 columns in that order, time
    starting at 5 min, 200 samples 0.1 min apart of waves whose period,
    phase and amplitude differ per cell, written with every digit."""
    import math
    from dense_b200 import workloads
    names = workloads.templates()["her_model_2014"]["species"]
    rng = np.random.Generator(np.random.PCG64(51))
    per = rng.uniform(1.5, 4.0, size=(2, 7))
    ph = rng.uniform(0.0, 2 * math.pi, size=(2, 7))
    amp = rng.uniform(1.0, 8.0, size=(2, 7))
    cols = ["pd", "mh1"]
    flags = ["1" if n in cols else "0" for n in names]
    lines = ["", "# exported trajectory (synthetic)", "cell-total, time-start, time-col, cell-start, cell-end, "
             "specie-option,", "10,5,0,0,7," + ",".join(flags) + ",", "", ",".join(cols) + ","]
    for k in range(200):
        t = 5.0 + 0.1 * k
        for c in range(7):
            v = [20.0 + amp[j, c] * math.sin(2 * math.pi * t / per[j, c] + ph[j, c]) + 0.01 * rng.normal()
                 for j in range(2)]
            lines.append(",".join(repr(float(x)) for x in v) + ",")
        lines.append("")
    with open(os.path.join(HERE, "inputs", "her_traj_waves.csv"), "w") as f:
        f.write("\n".join(lines) + "\n")


def import_samples(name):
    """(header, samples [k][species][cells], species names) of an import case."""
    from dense_b200 import csvio, workloads
    names = workloads.templates()["her_model_2014"]["species"]
    case = IMPORT_CASES[name]
    head, x = csvio.read_trajectory(open(os.path.join(HERE, case["file"])).read(), names)
    k = min(int(np.ceil(case["minutes"] / case["interval"])), x.shape[0])
    return head, x[:k], names


def run_import(name):
    from oracle.pyoracle import load_ref
    case = IMPORT_CASES[name]
    head, x, names = import_samples(name)
    R = load_ref("her_model_2014")
    cells = head["cell_total"]
    nprm = R.num_params
    sim = R.create(np.zeros(cells + 1, np.int32), np.zeros(1, np.int32), np.zeros((cells, nprm)), np.zeros(nprm),
                   None, case["interval"])
    for a in case["analyses"]:
        sp = [names.index(n) for n in a["species"]]
        if a["kind"] == "basic":
            sim.add_basic(sp, a["cells"][0], a["cells"][1], a["t"][0], a["t"][1])
        else:
            sim.add_oscillation(sp, a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"], a["intvl"])
    out = {"chunks": sim.replay(x, head["time_start"], case["interval"]), "status": np.int32(sim.status())}
    for i, a in enumerate(case["analyses"]):
        if a["kind"] == "basic":
            b = sim.basic(i)
            for k in ("mins", "sums", "maxs", "samples", "time", "cell_mins", "cell_sums", "cell_maxs"):
                out["a%d_%s" % (i, k)] = np.asarray(b[k])
        else:
            o = sim.oscillation(i)
            for k in ("amps", "pers", "avg_peak", "ncrit", "samples", "time"):
                out["a%d_%s" % (i, k)] = np.asarray(o[k])
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **out)
    print("ref_%s.npz" % name, len(out), "arrays")


if __name__ == "__main__":
    # no arguments: the CTest files, the command-line cases and every small
    # case; names (from CASES or FULL_CASES) regenerate just those fixtures
    if len(sys.argv) > 1:
        for name in sys.argv[1:]:
            run_import(name) if name in IMPORT_CASES else run_ref(name)
    else:
        copy_ctest()
        copy_inputs()
        write_waves_trajectory()
        run_cli_cases()
        for name in CASES:
            run_ref(name)
        for name in IMPORT_CASES:
            run_import(name)
