"""FP32+Kahan against FP64 on the batched her_model_2014 workload.

Runs the same seeded sets (template parameters x exp(U(ln .5, ln 2)), 200
cells, dt 0.01 min, Oscillation of mh1 over every cell every 0.1 min) in
both precisions and reports, per set, the relative difference of the mean
oscillation period and amplitude (sets where FP64 finds both finite) and of
the final state; prints one JSON object.

  python -m dense_b200.precision_check [--sets N] [--minutes M] [--window W]
"""

import argparse
import json
import time

import numpy as np

from . import engine as E
from . import workloads


def compare(num_sets=512, minutes=1200.0, window=float("inf"), seed=2, device=0):
    """`window`: the Oscillation analysis covers [0, window) minutes."""
    sets = workloads.log_uniform_sets(num_sets, cells=200, width=4, duration=minutes, seed=seed)
    an = [E.Analysis.oscillation(workloads.her_species("mh1"), 0, 200, 0.0, window, 4.0, 0.1)]
    out = {}
    for name, prec in (("fp64", E.FP64), ("fp32", E.FP32_KAHAN)):
        b = E.Batch("her_model_2014", sets, 0.01, 0.1, an, precision=prec, device=device)
        t0 = time.perf_counter()
        b.run()
        b.sync()
        secs = time.perf_counter() - t0
        per = np.full(num_sets, np.nan)
        amp = np.full(num_sets, np.nan)
        state = []
        for i in range(num_sets):
            o = b.oscillation(0, i)
            with np.errstate(invalid="ignore"):
                if np.isfinite(o["pers"][0]).any():
                    per[i] = np.nanmean(o["pers"][0])
                if np.isfinite(o["amps"][0]).any():
                    amp[i] = np.nanmean(o["amps"][0])
            state.append(b.state(i))
        out[name] = dict(per=per, amp=amp, state=np.array(state), seconds=secs,
                         cell_steps=b.info()["total_cell_steps"])
        b.close()
    a, f = out["fp64"], out["fp32"]
    ok = np.isfinite(a["per"]) & np.isfinite(f["per"]) & np.isfinite(a["amp"]) & np.isfinite(f["amp"])
    rp = np.abs(f["per"][ok] - a["per"][ok]) / np.abs(a["per"][ok])
    ra = np.abs(f["amp"][ok] - a["amp"][ok]) / np.maximum(np.abs(a["amp"][ok]), 1e-12)
    fin = np.isfinite(a["state"]) & np.isfinite(f["state"])
    rs = np.abs(f["state"][fin] - a["state"][fin]) / np.maximum(np.abs(a["state"][fin]), 1e-3)

    def stats(x):
        return {"median": float(np.median(x)), "p99": float(np.quantile(x, 0.99)), "max": float(np.max(x))} \
            if x.size else None

    return {"sets": num_sets, "minutes": minutes, "window": window, "sets_compared": int(ok.sum()),
            "period_rel": stats(rp), "amplitude_rel": stats(ra), "final_state_rel": stats(rs),
            "oscillation_found_mismatch": int((np.isfinite(a["per"]) != np.isfinite(f["per"])).sum()),
            "fp64_cell_steps_per_s": a["cell_steps"] / a["seconds"],
            "fp32_cell_steps_per_s": f["cell_steps"] / f["seconds"]}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--sets", type=int, default=512)
    ap.add_argument("--minutes", type=float, default=1200.0)
    ap.add_argument("--window", type=float, default=float("inf"), help="Oscillation window end (minutes)")
    a = ap.parse_args(argv)
    print(json.dumps(compare(a.sets, a.minutes, a.window)))


if __name__ == "__main__":
    main()
