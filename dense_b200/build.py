"""Build recipe of the engine libraries (one per DENSE model).

Each library is compiled for sm_100a only, in-tree, into
``dense_b200/_lib/libdense_b200_<model>.so``:

* ``kernels_fp64.cu`` with ``--fmad=false`` (no FMA contraction, so the FP64
  engine rounds every multiply and add like DENSE's x86-64 build);
* ``kernels_fp32.cu`` (FP32 rates, Kahan-compensated state);
* ``engine_api.cu``, the host set-up and the C ABI of include/dense_b200.h.

The model headers come from the model directory inside the DENSE tree
named by $DENSE_REF_DIR (dense_b200.models).  When the variable is unset
but a library was built before, the prebuilt library is used as is.
"""

import concurrent.futures as cf
import os
import subprocess

from .models import MODEL_DIRS, model_dir

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
ENGINE = os.path.join(CSRC, "engine")
API = os.path.join(CSRC, "model_api")
INCLUDE = os.path.join(ROOT, "include")
LIB_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(HERE, "_lib", "obj")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
          "--expt-relaxed-constexpr"]

UNITS = {
    "kernels_fp64.cu": ["--fmad=false"],
    "kernels_fp32.cu": [],
    "engine_api.cu": [],
    "noalloc.cu": ["--fmad=false"],
}


def lib_path(model):
    return os.path.join(LIB_DIR, "libdense_b200_%s.so" % model)


def _sources():
    out = [os.path.join(ENGINE, f) for f in os.listdir(ENGINE)]
    out += [os.path.join(API, "dense_model_api.hpp"), os.path.join(INCLUDE, "dense_b200.h")]
    return out


def _up_to_date(target, deps):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d))


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n%s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr[-6000:]))
    return r.stdout + r.stderr


def build_model(model, force=False, verbose=False):
    out = lib_path(model)
    mdir = model_dir(model, required=not os.path.exists(out))
    if mdir is None or not os.path.isdir(mdir):
        if os.path.exists(out):
            return out
        raise RuntimeError("DENSE model directory %s not found and no prebuilt %s" % (mdir, out))
    deps = _sources() + [os.path.join(mdir, f) for f in os.listdir(mdir)]
    if not force and _up_to_date(out, deps):
        return out
    os.makedirs(OBJ_DIR, exist_ok=True)
    inc = ["-I", INCLUDE, "-I", API, "-I", mdir, "-I", ENGINE]
    objs = []
    jobs = []
    with cf.ThreadPoolExecutor(max_workers=3) as ex:
        for unit, flags in UNITS.items():
            obj = os.path.join(OBJ_DIR, "%s_%s.o" % (model, unit.replace(".cu", "")))
            objs.append(obj)
            cmd = [NVCC] + ARCH + COMMON + flags + inc + ["-Xptxas", "-v", "-c", os.path.join(ENGINE, unit), "-o", obj]
            jobs.append(ex.submit(_run, cmd))
        logs = [j.result() for j in jobs]
    _run([NVCC] + ARCH + ["-shared", "-o", out] + objs + ["-lcudart"])
    if verbose:
        print("\n".join(logs))
    return out


def cli_path(model):
    return os.path.join(LIB_DIR, "dense_simulation_%s" % model)


def build_cli(model, force=False):
    """DENSE's `simulation` command for the model, linked to its engine
    library (csrc/cli/simulation_main.cpp)."""
    lib = build_model(model, force)
    out = cli_path(model)
    src = os.path.join(CSRC, "cli", "simulation_main.cpp")
    if not force and _up_to_date(out, [src, lib, os.path.join(INCLUDE, "dense_b200.h")]):
        return out
    _run(["g++", "-O2", "-std=c++17", "-I", INCLUDE, src, "-o", out, "-L", LIB_DIR,
          "-l:" + os.path.basename(lib), "-Wl,-rpath,$ORIGIN"])
    return out


def csv_gen_path(model):
    return os.path.join(LIB_DIR, "dense_csv_gen_%s" % model)


def build_csv_gen(model, force=False):
    """DENSE's `csv_gen` for the model (csrc/cli/csv_gen_main.cpp): the
    parameter-file templates, from the engine library's model tables."""
    lib = build_model(model, force)
    out = csv_gen_path(model)
    src = os.path.join(CSRC, "cli", "csv_gen_main.cpp")
    if not force and _up_to_date(out, [src, lib, os.path.join(INCLUDE, "dense_b200.h")]):
        return out
    _run(["g++", "-O2", "-std=c++17", "-I", INCLUDE, src, "-o", out, "-L", LIB_DIR,
          "-l:" + os.path.basename(lib), "-Wl,-rpath,$ORIGIN"])
    return out


def build_all(models=None, force=False):
    out = {}
    for m in (models or MODEL_DIRS):
        out[m] = build_model(m, force)
        build_cli(m, force)
        build_csv_gen(m, force)
    return out
