"""The drop-in `simulation` command's argument and input checks, which all
run before the engine touches a GPU: each bad invocation exits 1 with a
message.  Where DENSE itself crashes on the same input (a missing -p or -d
file: segmentation fault; a partial parameter set: uncaught exception), the
command refuses it instead."""

import os
import subprocess

import pytest

from dense_b200.build import build_cli

HERE = os.path.dirname(os.path.abspath(__file__))
INPUTS = os.path.join(HERE, "golden", "inputs")
PARAMS = os.path.join(INPUTS, "her_param_sets.csv")
BASE = ["-c", "10", "-w", "5", "-t", "10", "-s", "0.01", "-u", "0.1"]


@pytest.fixture(scope="module")
def cli():
    return build_cli("her_model_2014")


def _run(cli, args, cwd):
    r = subprocess.run([cli] + args, cwd=cwd, capture_output=True, text=True, timeout=60)
    return r.returncode, r.stdout + r.stderr


@pytest.mark.parametrize("args,msg", [
    (["-p", "/nonexistent/p.csv"] + BASE, "not found or open"),
    (["-p", PARAMS, "-d", "/nonexistent/d.csv"] + BASE, "not found or open"),
    (["-p", PARAMS, "-b", "/nonexistent/b.csv"] + BASE, "not found or open"),
    (["-p", PARAMS, "-a", "/nonexistent/a.xml"] + BASE, "could not read analysis file"),
    (["-p", PARAMS, "-f", "/nonexistent/g.graphml", "-t", "10", "-s", "0.01", "-u", "0.1"], "is invalid"),
    (["-p", PARAMS, "-c", "0", "-w", "5", "-t", "10", "-s", "0.01", "-u", "0.1"], "invalid cell total"),
    (["-p", PARAMS, "-c", "10", "-w", "11", "-t", "10", "-s", "0.01", "-u", "0.1"], "invalid cell total"),
    (["-p", PARAMS, "-c", "10", "-w", "5", "-t", "10", "-s", "0", "-u", "0.1"], "step-size"),
    (["-p", PARAMS, "-t", "10", "-s", "0.01", "-u", "0.1"], "cell-graph"),
    (["-c", "10"], "useless state"),
    (["-p", PARAMS, "-g", "grad.csv"] + BASE, "--gradients] is not supported"),
])
def test_bad_invocations_exit_1_with_a_message(cli, tmp_path, args, msg):
    rc, out = _run(cli, args, tmp_path)
    assert rc == 1 and msg in out, out


def test_partial_parameter_set(cli, tmp_path):
    bad = tmp_path / "partial.csv"
    bad.write_text("1,2,3,\n")
    rc, out = _run(cli, ["-p", str(bad)] + BASE, tmp_path)
    assert rc == 1 and "Partial set" in out, out


def test_malformed_graph_files(cli, tmp_path):
    """Graph files whose vertex ids are not numbers, or that hold no edges,
    are refused like missing ones."""
    bad = tmp_path / "bad.graphml"
    bad.write_text('<graphml><graph><edge source="n0" target="nx"/></graph></graphml>\n')
    empty = tmp_path / "empty.graphml"
    empty.write_text("<graphml><graph></graph></graphml>\n")
    for g in (bad, empty):
        rc, out = _run(cli, ["-p", PARAMS, "-f", str(g), "-t", "10", "-s", "0.01", "-u", "0.1"], tmp_path)
        assert rc == 1 and "is invalid" in out, out


def test_malformed_analysis_xml(cli, tmp_path):
    xml = tmp_path / "a.xml"
    xml.write_text("<analyses><anlys type=\"basic\"><species>mh1</species><cell-start>zero</cell-start>"
                   "<cell-end>4</cell-end><time-start>0</time-start><time-end>5</time-end>"
                   "<out-file>b.csv</out-file></anlys></analyses>")
    rc, out = _run(cli, ["-p", PARAMS, "-a", str(xml)] + BASE, tmp_path)
    assert rc == 1 and "malformed input" in out, out
