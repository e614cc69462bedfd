"""The drop-in boundary from a native caller: include/dense_b200.h compiles
as C and as C++, a program links the model library with the documented
link line, and the entry points that need no GPU work from it."""

import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++17")])
def test_c_and_cpp_callers_link_and_plan(tmp_path, compiler, std):
    from dense_b200.build import build_model
    lib = build_model("her_model_2014")
    src = os.path.join(ROOT, "tests", "native", "abi_caller.c")
    exe = str(tmp_path / "caller")
    cmd = [compiler, std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include")]
    cmd += ["-x", "c++"] if compiler == "g++" else []
    cmd += [src, "-x", "none", "-L", os.path.dirname(lib), "-l:" + os.path.basename(lib),
            "-Wl,-rpath," + os.path.dirname(lib), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stdout + out.stderr
    f = out.stdout.split()
    assert f[0] == "14" and f[1] == "45" and f[2] == "ph1"
    assert int(f[3]) > 0 and f[4] == "0" and f[5] == "1"   # register kernel, one dependency level
    assert f[6] == "1" and "outside the tissue" in out.stdout


@pytest.mark.parametrize("compiler,std", [("gcc", "-std=c99"), ("g++", "-std=c++17")])
def test_surrogate_header_compiles_and_links(tmp_path, compiler, std):
    """include/dense_b200_surrogate.h from C and C++: a program links the
    surrogate library and its argument checks answer without a GPU."""
    from dense_b200 import surrogate
    lib = surrogate.build()
    src = os.path.join(ROOT, "tests", "native", "surrogate_caller.c")
    exe = str(tmp_path / "surrogate_caller")
    cmd = [compiler, std, "-Wall", "-Werror", "-I", os.path.join(ROOT, "include")]
    cmd += ["-x", "c++"] if compiler == "g++" else []
    cmd += [src, "-x", "none", "-L", os.path.dirname(lib), "-l:" + os.path.basename(lib),
            "-Wl,-rpath," + os.path.dirname(lib), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    out = subprocess.run([exe], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0 and out.stdout.split() == ["4"], out.stdout + out.stderr
