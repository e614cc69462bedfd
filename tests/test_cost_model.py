"""The algorithmic cost per cell-step behind the benchmark's roofline,
counted rather than estimated: the model's own active_rate specialisations
run with a counting arithmetic type and a context that records each read
(tests/native/count_ops.cpp), at the template parameters and DENSE's ring
sizes (from the oracle)."""

import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _count(model, tmp_path, avg_neighbours, S, params):
    from dense_b200.models import model_dir
    mdir = model_dir(model, required=False)
    if mdir is None or not os.path.isdir(mdir):
        pytest.skip("DENSE model headers not present")
    exe = str(tmp_path / ("count_%s" % model))
    r = subprocess.run(["g++", "-O0", "-std=c++17", "-w", "-I", os.path.join(ROOT, "dense_b200", "csrc", "model_api"),
                        "-I", mdir, os.path.join(ROOT, "tests", "native", "count_ops.cpp"), "-o", exe],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([exe, repr(float(avg_neighbours))] + [str(int(x)) for x in S] +
                         [repr(float(x)) for x in params], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    add, mul, div, cmp, nbr, deltas, species, rows = (int(x) for x in out.stdout.split())
    return dict(add=add, mul=mul, div=div, cmp=cmp, nbr=nbr, deltas=deltas, species=species, rows=rows)


def test_her_cost_matches_the_benchmark_constants(tmp_path):
    sys.path.insert(0, ROOT)
    import bench
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    from oracle.pyoracle import load_oracle
    p = workloads.template_params()
    off, ids = default_graph(200, 4)
    deg = float(np.diff(off).mean())
    S, _ = load_oracle("her_model_2014").create(off, ids, np.tile(p, (200, 1)), p, None, 0.01).ring_sizes()
    c = _count("her_model_2014", tmp_path, deg, S, p)
    assert deg == 4.5 and c["species"] == 14 and c["deltas"] == 52 and c["nbr"] == 2
    assert c["div"] + c["nbr"] == 13                       # the 13 IEEE divisions of a her cell-step
    flops = c["add"] + c["mul"] + c["div"] + c["nbr"] * (deg + 1) + 2 * c["deltas"] + 2 * c["species"]
    assert flops == bench.FLOPS_PER_CELL_STEP
    assert 8 * (2 * c["species"] + c["rows"]) == bench.BYTES_PER_CELL_STEP


def test_turing_cost_matches_the_benchmark_constant(tmp_path):
    """Turing-Pattern: 4 species read and written; its neighbour averages
    read the rows of this step and the last, the same arrays, so they add
    no distinct bytes."""
    sys.path.insert(0, ROOT)
    import bench
    from dense_b200 import workloads
    p = workloads.template_params("turing")
    c = _count("turing", tmp_path, 6.0, [2, 2, 2, 2], p)
    assert c["species"] == 4 and c["nbr"] == 2 and c["rows"] == 2
    assert 8 * 2 * c["species"] == bench.TURING_BYTES_PER_CELL_STEP
