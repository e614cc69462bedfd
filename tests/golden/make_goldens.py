"""Generates the golden fixtures under tests/golden/.

1. ``dense_ctest/``: the blessed output files of DENSE's own CTest suite for
   the deterministic path, copied verbatim as data
   (test/her_model_2014/{anlys_basic_a,anlys_oscil,cell_width_test_anlys,
   total_time_test_anlys,total_time_test_01_anlys}.csv and
   test/Nan_Test/anlys_basic_a.csv).
2. ``ref_<case>.npz``: full-precision outputs of DENSE itself (compiled from
   its sources into oracle/_ref/ by oracle/build.py and driven through
   oracle/ref_harness.cpp) on the small cases of CASES below, together with
   the inputs they were computed from.  The GPU tests compare the engine
   with these on machines without the DENSE tree.

Usage: python tests/golden/make_goldens.py   (needs the DENSE tree)
"""

import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

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


def copy_ctest():
    out = os.path.join(HERE, "dense_ctest")
    os.makedirs(out, exist_ok=True)
    for dst, src in CTEST.items():
        shutil.copyfile(os.path.join(dense_dir(), src), os.path.join(out, dst))


def run_ref(name):
    from oracle.pyoracle import load_ref
    case = build_case(name)
    R = load_ref(case["model"])
    if R is None:
        raise RuntimeError("DENSE harness not built")
    out = {}
    for s, ps in enumerate(case["sets"]):
        sim = R.create(ps["off"], ps["ids"], ps["cell_params"], ps["set_params"], ps["init_conc"], case["dt"],
                       ps.get("perturb"))
        for a in case["analyses"]:
            if a["kind"] == "basic":
                sim.add_basic(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1])
            elif a["kind"] == "oscillation":
                sim.add_oscillation(a["species"], a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"],
                                    a["intvl"])
        out["chunks_%d" % s] = sim.run(ps["duration"], case["interval"])
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
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % name), **out)
    print("ref_%s.npz" % name, len(out), "arrays")


if __name__ == "__main__":
    copy_ctest()
    for name in (sys.argv[1:] or list(CASES)):
        run_ref(name)
