"""Build recipe for the oracle (test infrastructure only).

Three kinds of artefact, per DENSE model:

* ``oracle/_lib/libdense_oracle_<model>.so`` -- the CPU restatement
  (dense_oracle.cpp) compiled against the model's headers through the
  engine's model-API headers.  Built with plain ``-O2``: x86-64 without
  ``-march`` has no FMA, so every multiply and add rounds separately, as in
  DENSE's own build (CMakeLists.txt:18-22).
* ``oracle/_ref/libdense_ref_<model>.so`` -- DENSE itself: the sources of
  its deterministic path compiled where they lie in the DENSE tree, linked
  with ref_harness.cpp, which drives them through the oracle's C interface.
* ``oracle/_ref/<model>_simulation`` -- DENSE's own ``simulation`` CLI for
  the model (deterministic_main.cpp), for byte-level checks of its CSV
  output; ``oracle/_ref/<model>_csv_gen`` -- DENSE's ``csv_gen`` (the
  parameter-file templates), for the same check of ours.

The DENSE tree is ``$DENSE_REF_DIR``; ``use_default_tree`` points it at
the checkout this recipe was written for when the variable is unset and
that checkout exists.  When no tree is named (a machine that only runs the
prebuilt libraries) the reference builds are skipped.  Flags follow what DENSE needs to build with g++ 13:
``-include array -include fstream -include cstdint`` for headers it forgot,
``-DNDEBUG`` because the assert at sim/determ/determ.cpp:10 names an
undeclared variable, and ezxml compiled as C.

Usage: python oracle/build.py [model ...]
"""

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

from dense_b200.models import MODEL_DIRS, dense_dir, model_dir  # noqa: E402

LIB_DIR = os.path.join(HERE, "_lib")
REF_DIR = os.path.join(HERE, "_ref")
API_DIR = os.path.join(ROOT, "dense_b200", "csrc", "model_api")

REF_COMMON = [
    "core/build_once.cpp",
    "sim/base.cpp",
    "sim/determ/determ.cpp",
    "sim/determ/baby_cl.cpp",
    "utility/common_utils.cpp",
    "utility/color.cpp",
    "utility/preprocessor.cpp",
    "utility/numerics.cpp",
    "io/csvr.cpp",
    "io/csvw.cpp",
]
REF_CLI_EXTRA = [
    "deterministic_main.cpp",
    "io/arg_parse.cpp",
    "io/csvr_sim.cpp",
    "sim/stoch/fast_gillespie_direct_simulation.cpp",
    "sim/stoch/next_reaction_simulation.cpp",
    "sim/stoch/stoch.cpp",
]
REF_FLAGS = ["-O3", "-DNDEBUG", "-std=c++14", "-w",
             "-include", "array", "-include", "fstream", "-include", "cstdint"]


# the DENSE checkout this recipe reads when $DENSE_REF_DIR is unset
DEFAULT_TREE = "/root/reference"


def use_default_tree():
    """Set $DENSE_REF_DIR to DEFAULT_TREE when unset and that tree exists."""
    if not os.environ.get("DENSE_REF_DIR") and os.path.isdir(DEFAULT_TREE):
        os.environ["DENSE_REF_DIR"] = DEFAULT_TREE


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s%s" % (" ".join(cmd[:6]), r.stdout, r.stderr[-4000:]))


def _newer(target, sources):
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def oracle_lib_path(model):
    return os.path.join(LIB_DIR, "libdense_oracle_%s.so" % model)


def ref_lib_path(model):
    return os.path.join(REF_DIR, "libdense_ref_%s.so" % model)


def ref_cli_path(model):
    return os.path.join(REF_DIR, "%s_simulation" % model)


def ref_csv_gen_path(model):
    return os.path.join(REF_DIR, "%s_csv_gen" % model)


REF_CSV_GEN = ["csv_gen.cpp", "io/csvw.cpp", "io/csvr.cpp", "utility/color.cpp", "utility/common_utils.cpp",
               "utility/numerics.cpp"]


def build_oracle(model, force=False):
    """Compile the restatement for one model (needs the model headers)."""
    out = oracle_lib_path(model)
    mdir = model_dir(model, required=not os.path.exists(out))
    src = os.path.join(HERE, "dense_oracle.cpp")
    hdr = os.path.join(API_DIR, "dense_model_api.hpp")
    if mdir is None or not os.path.isdir(mdir):
        if os.path.exists(out):
            return out
        raise RuntimeError("model directory %s not found and no prebuilt %s" % (mdir, out))
    if not force and _newer(out, [src, hdr]):
        return out
    os.makedirs(LIB_DIR, exist_ok=True)
    _run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-w",
          "-I", API_DIR, "-I", mdir, src, "-o", out])
    return out


def _ezxml_obj():
    src = os.path.join(dense_dir(), "source", "io", "ezxml", "ezxml.c")
    obj = os.path.join(REF_DIR, "ezxml.o")
    if not _newer(obj, [src]):
        _run(["gcc", "-O3", "-fPIC", "-w", "-c", src, "-o", obj])
    return obj


def build_ref(model, force=False, cli=True):
    """Compile DENSE's own deterministic path for one model, if present."""
    tree = dense_dir(required=False)
    if tree is None:
        return None
    srcdir = os.path.join(tree, "source")
    mdir = model_dir(model)
    if not os.path.isdir(srcdir) or not os.path.isdir(mdir):
        return None
    os.makedirs(REF_DIR, exist_ok=True)
    inc = ["-I", mdir, "-I", srcdir]
    lib = ref_lib_path(model)
    harness = os.path.join(HERE, "ref_harness.cpp")
    if force or not _newer(lib, [harness]):
        srcs = [os.path.join(srcdir, s) for s in REF_COMMON]
        _run(["g++"] + REF_FLAGS + ["-fPIC", "-shared"] + inc + [harness] + srcs + ["-o", lib])
    if cli:
        exe = ref_cli_path(model)
        if force or not os.path.exists(exe):
            obj = _ezxml_obj()
            srcs = [os.path.join(srcdir, s) for s in REF_COMMON + REF_CLI_EXTRA]
            _run(["g++"] + REF_FLAGS + inc + srcs + [obj, "-o", exe])
        exe = ref_csv_gen_path(model)
        if force or not os.path.exists(exe):
            _run(["g++"] + REF_FLAGS + inc + [os.path.join(srcdir, s) for s in REF_CSV_GEN] + ["-o", exe])
    return lib


def build_all(models=None, force=False):
    models = models or list(MODEL_DIRS)
    built = {}
    for m in models:
        built[m] = (build_oracle(m, force), build_ref(m, force))
    return built


if __name__ == "__main__":
    use_default_tree()
    for m, (o, r) in build_all(sys.argv[1:] or None, force=True).items():
        print(m, o, r)
