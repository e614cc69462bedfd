"""DENSE model directories the engine is built for.

A DENSE model is compiled in: its four headers (specie_list.hpp,
reactions_list.hpp, reaction_deltas.hpp, model_impl.hpp) are included into
the engine's kernels at build time (DENSE does the same per model,
source/CMakeLists.txt:146-188).  Each entry maps a short model key to the
model directory inside a DENSE source tree.  The tree is named by the
environment variable DENSE_REF_DIR; there is no default, so a build never
picks up some other checkout by accident.  Without it, only libraries built
earlier can be used.
"""

import os

# key -> directory relative to the DENSE tree root
MODEL_DIRS = {
    "her_model_2014": "models/her_model_2014",
    "turing": "models/Turing-Pattern",
    "nan_test": "test/Nan_Test",
    "delay_reaction": "models/delay_reaction",
    "bz": "models/Belousov-Zhabotinksy",
    "briggs_rauscher": "models/briggs-rauscher",
}

ENV = "DENSE_REF_DIR"


def dense_dir(required=True):
    """The DENSE source tree named by $DENSE_REF_DIR.

    With required=False, None when the variable is unset or does not name
    a directory; otherwise that case raises an error naming the variable.
    """
    d = os.environ.get(ENV)
    if d and os.path.isdir(d):
        return d
    if not required:
        return None
    why = "is not set" if not d else "names %r, which is not a directory" % d
    raise RuntimeError("%s %s: set it to a DENSE source tree (the directory holding models/ and source/)"
                       % (ENV, why))


def model_dir(key, required=True):
    """The model's directory inside the DENSE tree (None when the tree is
    not named and required is False)."""
    d = dense_dir(required)
    return None if d is None else os.path.join(d, MODEL_DIRS[key])
