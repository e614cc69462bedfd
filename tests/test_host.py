"""Host-side logic that needs no GPU: the C ABI exports, CSV reading,
report formatting."""

import ctypes
import os
import re

import numpy as np
import pytest

from dense_b200 import csvio, report

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "dense_b200.h")).read()
    return sorted(set(re.findall(r"DENSE_API [a-z_ *]+?\b(dense_[a-z_]+)\(", text)))


@pytest.mark.parametrize("model", ["her_model_2014", "turing", "nan_test", "delay_reaction", "bz",
                                   "briggs_rauscher"])
def test_library_exports_every_declared_symbol(model):
    from dense_b200.build import build_model
    path = build_model(model)
    lib = ctypes.CDLL(path)
    syms = declared_symbols()
    assert len(syms) >= 17
    for s in syms:
        assert hasattr(lib, s), s


def test_surrogate_library_exports_every_declared_symbol():
    from dense_b200 import surrogate
    lib = ctypes.CDLL(surrogate.build())
    text = open(os.path.join(ROOT, "include", "dense_b200_surrogate.h")).read()
    names = sorted(set(re.findall(r"^int (dense_[a-z0-9_]+)\(", text, re.M)))
    assert len(names) == 15, names
    for name in names:
        assert hasattr(lib, name), name


def test_surrogate_entry_points_refuse_bad_arguments_on_the_host():
    """Shape and argument checks return 1 before any CUDA call (so they run
    without a GPU): rows not a positive multiple of 128, N outside [16, 256],
    K not a positive multiple of 64, a bias epilogue without a bias, too many cells for the
    synchrony kernel, bad encode and score arguments."""
    from dense_b200 import surrogate
    L = ctypes.CDLL(surrogate.build())
    vp, i, i64, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_int64, ctypes.c_double
    L.dense_mlp_gemm_ws.argtypes = [vp, i, vp, i, vp, i, i, i, i, i, vp, vp, i, vp, vp, ctypes.c_size_t, vp]
    p = vp(16)  # never dereferenced: every call below is refused first
    for M, N, K, epi, bias in ((100, 64, 64, 0, None), (0, 64, 64, 0, None), (128, 64, 0, 0, None),
                               (128, 8, 64, 0, None), (128, 512, 64, 0, None),
                               (128, 64, 96, 0, None), (128, 64, 64, 2, None), (128, 64, 64, 3, p)):
        assert L.dense_mlp_gemm_ws(p, K, p, K, p, N, M, N, K, epi, bias, p, N, p, None, 0, None) == 1
    L.dense_features_synchrony.argtypes = [vp, i64, i64, i, vp, i, vp, vp]
    assert L.dense_features_synchrony(p, 0, 0, 2048, p, 1, p, None) == 1
    L.dense_features_encode.argtypes = [vp, i, i, vp, vp, i, d, vp, i, i, vp]
    assert L.dense_features_encode(p, 45, 10, p, p, 80, 1.386, p, 64, 128, None) == 1   # k > in_pad
    assert L.dense_features_encode(p, 45, 200, p, p, 44, 1.386, p, 64, 128, None) == 1  # n > Bp
    L.dense_features_score.argtypes = [vp, i, i, i, vp, vp, d, d, d, d, d, vp, vp]
    assert L.dense_features_score(p, 10, 4, 1, p, p, 0.1, 30.0, 3.0, 50.0, 0.1, p, None) == 1  # nout < 5
    assert L.dense_features_score(p, 10, 5, 0, p, p, 0.1, 30.0, 3.0, 50.0, 0.1, p, None) == 1  # no networks


def test_model_info_matches_oracle():
    from dense_b200.engine import load
    from oracle.pyoracle import load_oracle
    for model in ("her_model_2014", "turing", "nan_test"):
        L = load(model)
        O = load_oracle(model)
        assert (L.num_species, L.num_reactions, L.num_delay_reactions, L.num_critical_species, L.num_params) == \
            (O.num_species, O.num_reactions, O.num_delay_reactions, O.num_critical_species, O.num_params)
        assert L.species == O.species and L.reactions == O.reactions
    L = load("her_model_2014")
    assert (L.num_species, L.num_reactions, L.num_delay_reactions, L.num_critical_species, L.num_params) == \
        (14, 34, 8, 3, 45)


def test_csv_trailing_value_rule():
    # a value is emitted only at a comma (io/csvr.cpp:80-99)
    assert csvio.read_reals("5.1, 5.2, 5.3, 5.9\n") == [5.1, 5.2, 5.3]
    assert csvio.read_reals("1,\n2,") == [1.0, 2.0]
    assert csvio.read_reals("1\n2,") == [12.0]


def test_csv_comments_and_headers():
    text = "# a comment, with commas\nname, other,\n1e-3, -2.5e2,+3,"
    assert csvio.read_reals(text) == [1e-3, -250.0, 3.0]


def test_csv_param_sets_partial_is_error():
    with pytest.raises(ValueError):
        csvio.read_param_sets("1,2,3,", 2)
    assert csvio.read_param_sets("1,2,3,4,", 2) == [[1.0, 2.0], [3.0, 4.0]]


def test_csv_init_conc_pads_and_truncates():
    assert csvio.read_init_conc("1,2,", 4) == [1.0, 2.0, 0.0, 0.0]
    assert csvio.read_init_conc("1,2,3,4,5,", 3) == [1.0, 2.0, 3.0]


def test_report_number_format():
    assert report.fmt(188.37427272) == "188.374"
    assert report.fmt(0.0) == "0"
    assert report.fmt(2999.9900000190623) == "2999.99"
    assert report.fmt(float("nan")) == "nan"
    assert report.fmt(-float("nan")) == "-nan"
    assert report.fmt(1e-7) == "1e-07"


def test_plan_kernels_and_bytes():
    """dense_engine_plan (no GPU): register kernel for unordered sets of at
    most 256 cells, memory kernel above that or on request, for ordered
    (Turing) sets a thread group the width of the widest dependency level
    per step in flight, hints checked."""
    from dense_b200 import tissue, workloads
    from dense_b200.engine import DenseError, ParameterSet, SCHEDULE_MEMORY, plan
    p = workloads.template_params()
    sets = []
    for n in (16, 256, 300, 1024):
        off, ids = tissue.default_graph(n, 4)
        sets.append(ParameterSet(off, ids, p, duration=100))
    off, ids = tissue.default_graph(200, 4)
    sets.append(ParameterSet(off, ids, p, duration=100, schedule=SCHEDULE_MEMORY))
    sets.append(ParameterSet(off, ids, p, duration=100, schedule=SCHEDULE_MEMORY, mem_block=96))
    nbytes, kernel, levels = plan("her_model_2014", sets, 0.01, 1.0)
    assert list(kernel) == [0, 0, 256, 256, 224, 96] and (levels == 1).all()
    assert (np.diff(nbytes[:4]) > 0).all() and nbytes[4] == nbytes[5]
    tp = workloads.template_params("turing")
    ts = []
    for N in (8, 16, 64):
        off, ids = tissue.default_graph(N * N, N)
        ts.append(ParameterSet(off, ids, tp, duration=10))
    _, kernel, levels = plan("turing", ts, 0.01, 1.0)
    # wave kernel: one warp per level, three steps in flight
    assert list(kernel) == [96, 96, 96] and (levels > 1).all()
    with pytest.raises(DenseError):
        plan("her_model_2014", [ParameterSet(off, ids, tp, duration=10)], 0.01, 1.0)
    off, ids = tissue.default_graph(200, 4)
    with pytest.raises(DenseError):
        plan("her_model_2014", [ParameterSet(off, ids, p, duration=10, mem_block=48)], 0.01, 1.0)


@pytest.mark.parametrize("model", ["her_model_2014", "turing", "nan_test", "delay_reaction", "bz",
                                   "briggs_rauscher"])
def test_csv_gen_matches_dense(model, tmp_path):
    """The drop-in csv_gen writes the same three template files, byte for
    byte, and the same console text as DENSE's csv_gen built from source."""
    import subprocess
    from dense_b200.build import build_csv_gen
    from oracle.build import ref_csv_gen_path
    ref = ref_csv_gen_path(model)
    if not os.path.exists(ref):
        pytest.skip("DENSE's csv_gen not built here")
    ours = build_csv_gen(model)
    outs = {}
    for name, exe in (("ref", ref), ("ours", ours)):
        d = tmp_path / name
        d.mkdir()
        r = subprocess.run([exe, str(d) + "/"], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0
        outs[name] = (r.stdout.replace(str(d), "DIR"),
                      {f: (d / f).read_bytes() for f in ("param_sets_template.csv", "param_pert_template.csv",
                                                          "param_grad_template.csv")})
    assert outs["ours"] == outs["ref"]
    r = subprocess.run([ours], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "Missing required command line argument" in r.stdout


def _levels(off, ids):
    """Dependency levels of DENSE's in-order sweep: a cell comes after every
    lower-numbered neighbour whose row of this step it reads."""
    n = len(off) - 1
    level = [0] * n
    for c in range(n):
        lv = [level[v] + 1 for v in ids[off[c]:off[c + 1]] if v < c]
        level[c] = max(lv) if lv else 0
    return max(level) + 1


def test_plan_levels_of_in_order_reads_on_irregular_tissues():
    """dense_engine_plan's dependency levels for Turing's in-order neighbour
    reads, on default grids and random graph-file tissues (0-12
    neighbours, self-loops), equal an independent count; without in-order
    reads (her_model_2014) a step is one level."""
    from dense_b200 import tissue, workloads
    from dense_b200.engine import ParameterSet, plan
    from tests.test_oracle import _random_tissue
    rng = np.random.Generator(np.random.PCG64(77))
    tp, hp = workloads.template_params("turing"), workloads.template_params()
    graphs = [tissue.default_graph(N * N, N) for N in (4, 8, 13)]
    graphs += [_random_tissue(rng, n, 12) for n in (1, 2, 30, 200)]
    for off, ids in graphs:
        _, _, lv = plan("turing", [ParameterSet(off, ids, tp, duration=1.0)], 0.01, 0.1)
        assert lv[0] == _levels(off, ids), (len(off) - 1, lv[0])
        _, _, lh = plan("her_model_2014", [ParameterSet(off, ids, hp, duration=1.0)], 0.01, 0.1)
        assert lh[0] == 1
