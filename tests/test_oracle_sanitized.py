"""The oracle under AddressSanitizer and UndefinedBehaviorSanitizer: built
from the same source with both sanitizers, it runs every golden case and
must report nothing and still reproduce DENSE's outputs bit for bit.

DENSE has no sanitizer builds of its own (its only checks are -Wall
-Werror and the NaN guards of sim/base.hpp:398-412); this covers the
test infrastructure the parity claims rest on.
"""

import os
import subprocess
import sys

import pytest

from tests.golden.cases import CASES, build_case

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
sys.path.insert(0, {root!r})
from oracle.pyoracle import OracleLib
from tests.helpers import load_fixture, mismatches, run_oracle
bad = []
for name, path in {cases!r}:
    got = run_oracle(OracleLib(path), name)
    m = mismatches(load_fixture(name), got)
    if m:
        bad.append((name, m[:3]))
print("MISMATCHES", bad)
sys.exit(1 if bad else 0)
"""


def _runtime(name):
    r = subprocess.run(["g++", "-print-file-name=" + name], capture_output=True, text=True)
    path = r.stdout.strip()
    return path if os.path.isabs(path) and os.path.exists(path) else None


def test_oracle_is_clean_under_asan_and_ubsan(tmp_path):
    from dense_b200.models import model_dir
    asan = _runtime("libasan.so")
    if asan is None:
        pytest.skip("no AddressSanitizer runtime for g++ here")
    api = os.path.join(ROOT, "dense_b200", "csrc", "model_api")
    src = os.path.join(ROOT, "oracle", "dense_oracle.cpp")
    libs = {}
    for name in sorted(CASES):
        model = build_case(name)["model"]
        if model in libs:
            continue
        mdir = model_dir(model, required=False)
        if mdir is None or not os.path.isdir(mdir):
            pytest.skip("DENSE model headers not present")
        out = str(tmp_path / ("liboracle_%s_san.so" % model))
        r = subprocess.run(["g++", "-O1", "-g", "-std=c++17", "-fPIC", "-shared", "-w", "-fno-omit-frame-pointer",
                            "-fsanitize=address,undefined", "-fno-sanitize-recover=undefined",
                            "-I", api, "-I", mdir, src, "-o", out], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-3000:]
        libs[model] = out
    cases = [(name, libs[build_case(name)["model"]]) for name in sorted(CASES)]
    env = dict(os.environ, LD_PRELOAD=asan, ASAN_OPTIONS="detect_leaks=0:abort_on_error=0",
               UBSAN_OPTIONS="print_stacktrace=1")
    r = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, cases=cases)], env=env,
                       capture_output=True, text=True, timeout=900)
    report = r.stdout[-2000:] + r.stderr[-4000:]
    assert r.returncode == 0, report
    assert "AddressSanitizer" not in r.stderr and "runtime error" not in r.stderr, report
    assert "MISMATCHES []" in r.stdout, report
