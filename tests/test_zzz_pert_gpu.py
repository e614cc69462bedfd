"""FP64 engine parity with -b perturbation factors: they resize DENSE's
rings (base.cpp:55-140), moving the rows that zero-truncated delays read
(lag S - 1).  The engine's run of the case is compared bit for bit with
DENSE's own outputs (tests/golden/ref_her_pert_factors.npz).  This file is
collected last."""

import pytest

from tests.golden.cases import build_case
from tests.helpers import load_fixture, mismatches, run_engine

pytestmark = pytest.mark.gpu


def test_fp64_bitwise_vs_dense_with_perturbation_factors():
    want = load_fixture("her_pert_factors")
    got = run_engine("her_pert_factors")
    for s in range(len(build_case("her_pert_factors")["sets"])):
        assert got["status_%d" % s] == 0
    assert mismatches(want, got) == []
