"""Analysis of an imported trajectory on the GPU (dense_engine_analyze_samples
and `simulation -i`): the engine's analyses over the samples of a trajectory
export -- one DENSE itself wrote, with a time column and its species in -o
order, and a synthetic one with uneven waves per cell, a later start time
and cells past the exported range -- equal, bit for bit, DENSE's own
BasicAnalysis and OscillationAnalysis over the same samples (fixtures of
tests/golden/make_goldens.py), and the command writes them as DENSE's show()
would."""

import os
import subprocess

import numpy as np
import pytest

from dense_b200 import engine as E, report
from dense_b200.build import build_cli
from tests.golden.make_goldens import IMPORT_CASES, import_samples
from tests.helpers import load_fixture, mismatches

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _analyses(case, names):
    out = []
    for a in case["analyses"]:
        sp = [names.index(n) for n in a["species"]]
        if a["kind"] == "basic":
            out.append(E.Analysis.basic(sp, a["cells"][0], a["cells"][1], a["t"][0], a["t"][1]))
        else:
            out.append(E.Analysis.oscillation(sp, a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"],
                                              a["intvl"]))
    return out


@pytest.mark.parametrize("name", sorted(IMPORT_CASES))
def test_engine_analyses_of_imported_samples_match_dense(name):
    case = IMPORT_CASES[name]
    head, x, names = import_samples(name)
    L = E.load("her_model_2014")
    cells = head["cell_total"]
    ps = E.ParameterSet(np.zeros(cells + 1, np.int32), np.zeros(1, np.int32), np.zeros(L.num_params),
                        duration=case["minutes"])
    b = E.Batch("her_model_2014", [ps], case["interval"], case["interval"], _analyses(case, names))
    b.analyze_samples(0, x, head["time_start"])
    chunks, _ = b.progress()
    got = {"chunks": chunks[0], "status": b.status()[0]}
    for i, a in enumerate(case["analyses"]):
        r = b.basic(i, 0) if a["kind"] == "basic" else b.oscillation(i, 0)
        for k, v in r.items():
            got["a%d_%s" % (i, k)] = np.asarray(v)
    b.close()
    assert mismatches(load_fixture(name), got) == []


@pytest.mark.parametrize("name", sorted(IMPORT_CASES))
def test_simulation_command_import_writes_dense_analysis_text(name, tmp_path):
    case = IMPORT_CASES[name]
    want = load_fixture(name)
    head, _, names = import_samples(name)
    xml = "<analyses>"
    for i, a in enumerate(case["analyses"]):
        xml += ("<anlys type=\"%s\"><species>%s</species><cell-start>%d</cell-start><cell-end>%d</cell-end>"
                "<time-start>%r</time-start><time-end>%r</time-end><out-file>out%d.csv</out-file>"
                % (a["kind"], ", ".join(a["species"]), a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], i))
        if a["kind"] == "oscillation":
            xml += "<win-range>%r</win-range><anlys-intvl>%r</anlys-intvl>" % (a["win"], a["intvl"])
        xml += "</anlys>"
    (tmp_path / "a.xml").write_text(xml + "</analyses>")
    r = subprocess.run([build_cli("her_model_2014"), "-i", os.path.join(GOLDEN, case["file"]), "-t",
                        repr(case["minutes"]), "-u", repr(case["interval"]), "-a", "a.xml"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    for i, a in enumerate(case["analyses"]):
        ids = [names.index(n) for n in a["species"]]
        res = {k[len("a%d_" % i):]: v for k, v in want.items() if k.startswith("a%d_" % i)}
        got = (tmp_path / ("out%d.csv" % i)).read_text()
        if a["kind"] == "oscillation":
            assert got == report.oscillation_csv(names, ids, res, a["cells"][0], a["cells"][1], a["t"][0])
            continue
        # BasicAnalysis::show indexes its per-species vectors by species id
        # (basic.ipp:69-72): rows of species whose id is past the observed
        # count are undefined in DENSE and nan here, in either sign
        text = report.basic_csv(names, ids, res, a["cells"][0], a["cells"][1], a["t"][0]).split("\n")
        lines = got.split("\n")
        assert len(lines) == len(text)
        undefined = {names[sp] for sp in ids if sp >= len(ids)}
        for g, w in zip(lines, text):
            if w.split(",")[0] in undefined:
                assert g.split(",")[0] == w.split(",")[0] and all(v in ("nan", "-nan") for v in g.split(",")[1:])
            else:
                assert g == w
