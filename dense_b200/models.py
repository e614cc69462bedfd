"""DENSE model directories the engine is built for.

A DENSE model is compiled in: its four headers (specie_list.hpp,
reactions_list.hpp, reaction_deltas.hpp, model_impl.hpp) are included into
the engine's kernels at build time (DENSE does the same per model,
source/CMakeLists.txt:146-188).  Each entry maps a short model key to the
model directory inside a DENSE source tree; the tree is found through
$DENSE_REF_DIR (default: the reference checkout this project was built
against, see __graft_entry__.build).
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

DEFAULT_DENSE_DIR = "/root/reference"


def dense_dir():
    return os.environ.get("DENSE_REF_DIR", DEFAULT_DENSE_DIR)


def model_dir(key):
    return os.path.join(dense_dir(), MODEL_DIRS[key])
