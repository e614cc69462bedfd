"""FP32+Kahan against FP64, per benchmark configuration.

Runs the same seeded inputs in both precisions and reports relative
differences |fp32 - fp64| / max(|fp64|, 1e-3) (final states, Basic
outputs) or |fp32 - fp64| / |fp64| (oscillation period and amplitude, where
FP64 finds both finite); prints one JSON object.

* ``batch`` (default): 512 her_model_2014 sets (template parameters x
  exp(U(ln .5, ln 2))), 200 cells, dt 0.01 min, Oscillation of mh1 over
  every cell every 0.1 min over [0, window); per-set mean period and
  amplitude and every final state.
* ``single``: one her_model_2014 set, 200 cells, every parameter of every
  cell x U(0.95, 1.05), 600 min, Basic over every species and cell and
  Oscillation of mh1 and ph1 over [0, window); per-cell outputs.
* ``mixed``: the first N sets of the uneven mixed batch (her_model_2014 and
  Turing-Pattern, horizons 100-1200 min), no analyses; final states.

  python -m dense_b200.precision_check [--config batch|single|mixed]
      [--sets N] [--minutes M] [--window W]
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
    rp = _rel(f["per"][ok], a["per"][ok], 0.0)
    ra = _rel(f["amp"][ok], a["amp"][ok], 1e-12)
    rs = _rel(f["state"], a["state"])
    return {"config": "batch", "sets": num_sets, "minutes": minutes, "window": window,
            "sets_compared": int(ok.sum()),
            "period_rel": _stats(rp), "amplitude_rel": _stats(ra), "final_state_rel": _stats(rs),
            "oscillation_found_mismatch": int((np.isfinite(a["per"]) != np.isfinite(f["per"])).sum()),
            "fp64_cell_steps_per_s": a["cell_steps"] / a["seconds"],
            "fp32_cell_steps_per_s": f["cell_steps"] / f["seconds"]}


def _stats(x):
    x = np.asarray(x, np.float64).ravel()
    return {"median": float(np.median(x)), "p99": float(np.quantile(x, 0.99)), "max": float(np.max(x))} \
        if x.size else None


def _rel(f, a, floor=1e-3):
    f, a = np.asarray(f, np.float64), np.asarray(a, np.float64)
    ok = np.isfinite(f) & np.isfinite(a)
    return np.abs(f[ok] - a[ok]) / np.maximum(np.abs(a[ok]), floor)


def _run_both(model, sets, analyses, device, read):
    out = {}
    for name, prec in (("fp64", E.FP64), ("fp32", E.FP32_KAHAN)):
        b = E.Batch(model, sets, 0.01, 0.1, analyses, precision=prec, device=device)
        t0 = time.perf_counter()
        b.run()
        b.sync()
        secs = time.perf_counter() - t0
        out[name] = read(b)
        out[name]["seconds"] = secs
        out[name]["cell_steps"] = b.info()["total_cell_steps"]
        b.close()
    return out


def compare_single(minutes=600.0, window=float("inf"), device=0):
    """One perturbed her_model_2014 set (200 cells): final state, Basic and
    per-cell oscillation outputs."""
    s = workloads.perturbed_set(cells=200, width=4, duration=minutes, seed=1)
    nsp = len(workloads.templates()["her_model_2014"]["species"])
    an = [E.Analysis.basic(list(range(nsp)), 0, 200),
          E.Analysis.oscillation(workloads.her_species("mh1", "ph1"), 0, 200, 0.0, window, 4.0, 0.1)]

    def read(b):
        bs, o = b.basic(0, 0), b.oscillation(1, 0)
        return {"state": b.state(0), "basic": np.concatenate([bs["cell_mins"].ravel(), bs["cell_maxs"].ravel(),
                                                               bs["cell_sums"].ravel()]),
                "pers": o["pers"], "amps": o["amps"]}

    r = _run_both("her_model_2014", [s], an, device, read)
    a, f = r["fp64"], r["fp32"]
    both = np.isfinite(a["pers"]) & np.isfinite(f["pers"]) & np.isfinite(a["amps"]) & np.isfinite(f["amps"])
    return {"config": "single", "minutes": minutes, "window": window,
            "final_state_rel": _stats(_rel(f["state"], a["state"])),
            "basic_rel": _stats(_rel(f["basic"], a["basic"])),
            "cells_compared": int(both.sum()),
            "period_rel": _stats(_rel(f["pers"][both], a["pers"][both], 0.0)),
            "amplitude_rel": _stats(_rel(f["amps"][both], a["amps"][both], 1e-12)),
            "oscillation_found_mismatch": int((np.isfinite(a["pers"]) != np.isfinite(f["pers"])).sum())}


def compare_mixed(num_sets=512, device=0):
    """The first `num_sets` sets of the uneven mixed batch: final states, per model."""
    sets = workloads.mixed_sets(num_sets)
    res = {"config": "mixed", "sets": num_sets}
    for model, ss in sets.items():
        if not ss:
            continue
        r = _run_both(model, ss, (), device, lambda b: {"state": np.concatenate(
            [b.state(i).ravel() for i in range(len(b.sets))])})
        a, f = r["fp64"], r["fp32"]
        res[model] = {"sets": len(ss), "final_state_rel": _stats(_rel(f["state"], a["state"])),
                      "fp64_cell_steps_per_s": a["cell_steps"] / a["seconds"],
                      "fp32_cell_steps_per_s": f["cell_steps"] / f["seconds"]}
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=("batch", "single", "mixed"), default="batch")
    ap.add_argument("--sets", type=int, default=512)
    ap.add_argument("--minutes", type=float, default=None)
    ap.add_argument("--window", type=float, default=float("inf"), help="Oscillation window end (minutes)")
    a = ap.parse_args(argv)
    if a.config == "single":
        out = compare_single(a.minutes or 600.0, a.window)
    elif a.config == "mixed":
        out = compare_mixed(a.sets)
    else:
        out = compare(a.sets, a.minutes or 1200.0, a.window)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
