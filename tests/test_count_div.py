"""The engines' correctly rounded division by a neighbour count
(csrc/engine/count_div.cuh) equals IEEE division, checked on the host."""

import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ENGINE = os.path.join(os.path.dirname(HERE), "dense_b200", "csrc", "engine")


def test_div_by_count_matches_ieee_division(tmp_path):
    exe = str(tmp_path / "count_div_check")
    r = subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", ENGINE,
                        os.path.join(HERE, "native", "count_div_check.cpp"), "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr[-3000:])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-3000:]
    for line in out.stdout.splitlines():
        name, cases, fast = line.split()
        assert int(cases) > 8_000_000
        # the proof accepts the refined quotient for nearly every operand
        assert float(fast) > 0.99, line
