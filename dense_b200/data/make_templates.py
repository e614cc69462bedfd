"""Writes templates.json: each model's template parameter set (the first
set of the model directory's param_sets.csv) and initial concentrations
(init_conc.csv, where the model ships one), read with DENSE's CSV rules
(dense_b200.csvio).  The synthetic workloads start from these values.

Usage: python -m dense_b200.data.make_templates   (needs the DENSE tree)
"""

import json
import os

from dense_b200 import csvio
from dense_b200.models import MODEL_DIRS, model_dir

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "templates.json")


def main():
    from dense_b200.engine import load
    out = {}
    for key in MODEL_DIRS:
        d = model_dir(key)
        L = load(key)
        entry = {"num_params": L.num_params, "species": L.species, "reactions": L.reactions}
        for fname in ("param_sets.csv", "param_set.csv"):
            p = os.path.join(d, fname)
            if os.path.exists(p):
                sets = csvio.read_param_sets(open(p).read(), L.num_params)
                entry["params"] = sets[0] if sets else None
                break
        p = os.path.join(d, "init_conc.csv")
        if os.path.exists(p):
            entry["init_conc"] = csvio.read_init_conc(open(p).read(), L.num_species)
        out[key] = entry
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
