"""Analysis of an imported trajectory (`simulation -i`), on the CPU: the
trajectory reader, the command's refusals (before any GPU work), and the
oracle restatement's replay of the imported samples against DENSE's own
analyses over them (fixtures made by tests/golden/make_goldens.py with
DENSE's BasicAnalysis and OscillationAnalysis, oracle_replay of
oracle/ref_harness.cpp)."""

import os
import subprocess

import numpy as np
import pytest

from dense_b200 import csvio, workloads
from dense_b200.build import build_cli
from tests.golden.make_goldens import IMPORT_CASES, import_samples
from tests.helpers import load_fixture, mismatches

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")
NAMES = workloads.templates()["her_model_2014"]["species"]
EXPORT = os.path.join(GOLDEN, "cli", "her_traj_export_v", "traj.csv")


def test_reader_maps_columns_by_name_and_skips_the_time_column():
    """DENSE's export writes its species in the -o order (ph1, mh1, md here)
    with a Time column; the reader places every value under its species and
    cell and leaves what the file does not hold NaN."""
    head, x = csvio.read_trajectory(open(EXPORT).read(), NAMES)
    assert head["cell_total"] == 12 and head["time_col"] == 1 and (head["cell_start"], head["cell_end"]) == (0, 12)
    assert [NAMES[i] for i in head["species"]] == ["ph1", "mh1", "md"]
    assert x.shape == (300, len(NAMES), 12)
    rows = [ln for ln in open(EXPORT).read().splitlines() if ln.startswith(",") or ln.startswith("Time:")]
    last = rows[-1].split(",")
    assert x[-1, NAMES.index("ph1"), 11] == float(last[1]) and x[-1, NAMES.index("md"), 11] == float(last[3])
    held = set(head["species"])
    assert all(np.isnan(x[:, sp]).all() for sp in range(len(NAMES)) if sp not in held)


def test_reader_refuses_malformed_files():
    good = open(EXPORT).read()
    with pytest.raises(ValueError):
        csvio.read_trajectory("1,2,3,\n", NAMES)
    with pytest.raises(ValueError):
        csvio.read_trajectory(good.replace("Time,ph1,mh1,md,", "Time,ph1,pd,md,"), NAMES)   # column not flagged
    lines = good.splitlines()
    k = next(i for i, ln in enumerate(lines) if ln.startswith(",") and ln.count(",") == 4)
    lines[k] = ",1.5,oops,2,"
    with pytest.raises(ValueError):
        csvio.read_trajectory("\n".join(lines), NAMES)


@pytest.mark.parametrize("name", sorted(IMPORT_CASES))
def test_oracle_replay_matches_dense_analyses(name):
    from oracle.pyoracle import load_oracle
    case = IMPORT_CASES[name]
    head, x, names = import_samples(name)
    O = load_oracle("her_model_2014")
    cells = head["cell_total"]
    sim = O.create(np.zeros(cells + 1, np.int32), np.zeros(1, np.int32), np.zeros((cells, O.num_params)),
                   np.zeros(O.num_params), None, case["interval"])
    for a in case["analyses"]:
        sp = [names.index(n) for n in a["species"]]
        if a["kind"] == "basic":
            sim.add_basic(sp, a["cells"][0], a["cells"][1], a["t"][0], a["t"][1])
        else:
            sim.add_oscillation(sp, a["cells"][0], a["cells"][1], a["t"][0], a["t"][1], a["win"], a["intvl"])
    got = {"chunks": sim.replay(x, head["time_start"], case["interval"]), "status": np.int32(sim.status())}
    for i, a in enumerate(case["analyses"]):
        r = sim.basic(i) if a["kind"] == "basic" else sim.oscillation(i)
        for k, v in r.items():
            got["a%d_%s" % (i, k)] = np.asarray(v)
    assert mismatches(load_fixture(name), got) == []


@pytest.fixture(scope="module")
def cli():
    return build_cli("her_model_2014")


@pytest.mark.parametrize("args,msg", [
    (["-i", "/nonexistent/t.csv", "-t", "10", "-u", "0.1"], "not found or open"),
    (["-i", EXPORT, "-u", "0.1"], "No time-total or anlys-intvl"),
    (["-i", os.path.join(GOLDEN, "inputs", "her_param_sets.csv"), "-t", "10", "-u", "0.1"],
     "not a trajectory export"),
])
def test_import_refusals(cli, tmp_path, args, msg):
    r = subprocess.run([cli] + args, cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and msg in r.stdout, r.stdout


def test_import_refuses_analyses_the_file_cannot_feed(cli, tmp_path):
    """An analysis of a species the file does not hold, or of cells outside
    the exported range, is refused (DENSE's reader would throw from
    std::map::at / vector::at)."""
    def xml(species, c0, c1):
        p = tmp_path / ("a_%s_%d.xml" % (species, c1))
        p.write_text("<analyses><anlys type=\"basic\"><species>%s</species><cell-start>%d</cell-start>"
                     "<cell-end>%d</cell-end><time-start>0</time-start><time-end>5</time-end>"
                     "<out-file>b.csv</out-file></anlys></analyses>" % (species, c0, c1))
        return str(p)
    waves = os.path.join(GOLDEN, "inputs", "her_traj_waves.csv")   # 10 cells, 0-6 exported
    for f, x, msg in ((EXPORT, xml("pd", 0, 4), "holds no pd"), (waves, xml("mh1", 0, 9), "outside the imported")):
        r = subprocess.run([cli, "-i", f, "-t", "10", "-u", "0.1", "-a", x], cwd=tmp_path,
                           capture_output=True, text=True, timeout=60)
        assert r.returncode == 1 and msg in r.stdout, r.stdout
