"""The drop-in `simulation` command (dense_simulation_<model>): the files it
writes are byte-identical to those DENSE's own command writes for the same
arguments (tests/golden/cli, made by tests/golden/make_goldens.py with
DENSE built from its sources)."""

import os
import shlex
import subprocess

import pytest

from dense_b200.build import build_cli
from tests.golden.make_goldens import CLI_CASES

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


# Rows DENSE prints from past the end of its per-species vectors are kept
# in the fixtures as "undefined" (tests/golden/make_goldens.py); the engine
# prints nan on those rows, and every other byte must match.
@pytest.mark.parametrize("name", sorted(CLI_CASES))
def test_cli_output_files_match_dense(name, tmp_path):
    model, args, outs = CLI_CASES[name]
    exe = build_cli(model)
    cmd = [exe] + shlex.split(args.format(**{"in": os.path.join(GOLDEN, "inputs")}))
    r = subprocess.run(cmd, cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    for f in outs:
        want = open(os.path.join(GOLDEN, "cli", name, f), "rb").read()
        got = open(os.path.join(tmp_path, f), "rb").read()
        if b",undefined," not in want:
            assert got == want, f
            continue
        got_lines, want_lines = got.split(b"\n"), want.split(b"\n")
        assert len(got_lines) == len(want_lines), f
        for g, w in zip(got_lines, want_lines):
            if w.endswith(b",undefined,undefined,undefined"):
                assert g.split(b",")[0] == w.split(b",")[0] and g.count(b"nan") == 3, (f, g)
            else:
                assert g == w, (f, g, w)


def test_cli_several_sets_write_numbered_files(tmp_path):
    """With more than one parameter set every analysis writes x_####.y files
    (run_simulation.hpp:54-63, 113-121)."""
    exe = build_cli("her_model_2014")
    src = open(os.path.join(GOLDEN, "inputs", "her_param_sets.csv")).read()
    two = os.path.join(tmp_path, "two_sets.csv")
    row = [ln for ln in src.splitlines() if ln.strip() and not ln.startswith("#")][0]
    open(two, "w").write(row + "\n" + row + "\n")
    xml = os.path.join(tmp_path, "a.xml")
    open(xml, "w").write("<analyses><anlys type=\"basic\"><species>mh1</species><cell-start>0</cell-start>"
                         "<cell-end>4</cell-end><time-start>0</time-start><time-end>5</time-end>"
                         "<out-file>b.csv</out-file></anlys></analyses>")
    r = subprocess.run([exe, "-p", two, "-c", "8", "-w", "4", "-t", "5", "-u", "0.5", "-s", "0.01", "-a", xml],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout
    a = open(os.path.join(tmp_path, "b_0000.csv")).read()
    b = open(os.path.join(tmp_path, "b_0001.csv")).read()
    assert a == b and a.startswith("# Showing cells 0-4 until 4.5 min\n")
