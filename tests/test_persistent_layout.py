"""The persistent tensor-core GEMM's shared-memory layout
(csrc/surrogate/umma_gemm_persistent.cuh, persistent_smem), checked on the
host for the surrogate's shapes: it fits, stays aligned and keeps its ring
depth."""

import os
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(os.path.dirname(HERE), "dense_b200", "csrc", "surrogate")


def test_persistent_gemm_layouts_fit_and_stay_aligned(tmp_path):
    exe = str(tmp_path / "persistent_layout_check")
    r = subprocess.run([os.environ.get("NVCC", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17",
                        "-I", SRC, os.path.join(HERE, "native", "persistent_layout_check.cu"), "-o", exe],
                       capture_output=True, text=True)
    if r.returncode != 0:
        pytest.fail(r.stderr[-3000:])
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout[-3000:]
    assert out.stdout.count("ok ") == 24
