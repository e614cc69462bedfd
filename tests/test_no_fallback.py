"""The product path has no CPU fallback: without a GPU every entry point
that would compute fails loudly, and no module of the package refers to the
oracle (which only tests, smoke() and the benchmark's CPU baseline use)."""

import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_package_never_refers_to_the_oracle():
    pkg = os.path.join(ROOT, "dense_b200")
    hits = []
    for d, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".hpp", ".h")):
                text = open(os.path.join(d, f), errors="replace").read()
                if re.search(r"\boracle\b", text):
                    hits.append(os.path.relpath(os.path.join(d, f), ROOT))
    assert hits == []


def test_engine_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dense_b200 import engine as E, workloads
    s = workloads.perturbed_set(cells=8, width=4, duration=1.0)
    with pytest.raises(E.DenseError, match="(?i)cuda"):
        E.Batch("her_model_2014", [s], 0.01, 0.1)


def test_surrogate_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dense_b200.surrogate import MLP
    with pytest.raises(Exception):
        MLP(44, 5)
    from dense_b200 import search as S
    with pytest.raises(Exception):
        S.simulate_features(np.tile(S.template(), (2, 1)), cells=8)


def test_sharded_simulation_fails_loudly_without_a_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dense_b200 import engine as E, workloads
    from dense_b200.sharding import simulate_sharded
    s = workloads.perturbed_set(cells=8, width=4, duration=1.0)
    with pytest.raises(E.DenseError):
        simulate_sharded("her_model_2014", [s, s], 0.01, 0.1)
