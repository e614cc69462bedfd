"""Benchmark: cell-steps/s of the FP64 engine on her_model_2014.

Workload (the batched configuration): 4096 parameter sets, each template
parameter scaled by exp(U(ln 0.5, ln 2)) per set (seeded), 200 cells per set
on DENSE's default hexagonal tissue (-c 200 -w 4), dt 0.01 min, 1200 min,
Oscillation of mh1 over every cell sampled every 0.1 min (4-minute window).
A cell-step is one forward-Euler step of one cell of one set.

A timed step is one launch of the step kernel that advances every set by
1200/K minutes (K = --steps), so K steps cover the whole horizon; W warm-up
launches run first on the same batch, which is then reset (outside the
timed region).  The batch's history rings and oscillation windows total
well over the 126 MB L2, so no flush is needed between steps.

e2e: the same metric through the public API with host buffers: building the
batch from host arrays (host->device copies), the full horizon, and reading
every set's oscillation amplitude/period back to the host; the median of
--e2e-steps such passes (each one's time is in the line).

Multi-GPU (torchrun): each rank runs its own batch (sets shard with no
exchange; scaling is weak); times are the max over ranks.

--impl reference: DENSE's own deterministic path (compiled from its sources
into oracle/_ref by oracle/build.py) on every host core, each step a bounded
sample of the same workload.

Other workloads (--workload; each prints the same JSON keys):
  single  one her_model_2014 set of 200 cells, every parameter of every cell
          x U(0.95, 1.05), 600 min, Basic + Oscillation (a step = the run);
  mixed   10,000 her_model_2014 and Turing-Pattern sets of uneven size and
          horizon in one captured graph, autotuned schedules;
  turing  sets of one Turing-Pattern N x N grid (--grid), the wave kernel.
"""

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# Algorithmic cost of one her_model_2014 cell-step (FP64) at the template
# parameters, counted by evaluating the model's own rates with a counting
# arithmetic type (tests/native/count_ops.cpp, checked by
# tests/test_cost_model.py):
#  bytes: the lag-0 state read (14 x 8) and written (14 x 8) plus the 10
#         distinct history rows the rates read (pd at two lags, ph11 and
#         ph713 at three each, md, mh13) = 304 B;
#  flops: 34 rates (10 add, 45 mul, 11 div), two neighbour averages (4.5
#         adds and a division each on the 200-cell width-4 tissue), 52 delta
#         terms (mul + add) and 14 Euler updates (mul + add) = 209.
BYTES_PER_CELL_STEP = 304
FLOPS_PER_CELL_STEP = 209
DRAM_BYTES_PER_CELL_STEP = 16.4

METRIC = "cell-steps/s (FP64 plain)"


def batch_workload(num_sets, minutes, with_analyses):
    """The batched workload's name, the same in both arms' JSON lines."""
    return ("her_model_2014: %d parameter sets (template x exp(U(ln .5, ln 2)) per set), 200 cells each "
            "(-c 200 -w 4), dt 0.01 min, %g min, %s"
            % (num_sets, minutes, "Oscillation(mh1, all cells, window 4 min) every 0.1 min" if with_analyses
               else "no analyses"))


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        if "hbm_gbs" in d:
            return float(d["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs): frac is of measured"
    return 6650.0, "fallback 6650 GB/s (no measured peak file): frac is of fallback"


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, gpu):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_workload(num_sets, minutes, seed):
    from dense_b200 import workloads
    sets = workloads.log_uniform_sets(num_sets, cells=200, width=4, duration=minutes, seed=seed)
    return sets, workloads.batch_analyses(200, 0.1)


PARITY_FIXTURE = os.path.join("tests", "golden", "ref_her_cfg2_full.npz")


def batch_parity(batch):
    """The timed run's own results for the workload's sets that DENSE itself
    simulated into PARITY_FIXTURE (same seeds, 200 cells, 1200 min,
    Oscillation of mh1): final state and oscillation outputs, bit for bit."""
    path = os.path.join(ROOT, PARITY_FIXTURE)
    if not os.path.exists(path):
        return {"fixture": PARITY_FIXTURE, "checked": False, "why": "fixture missing"}
    want = dict(np.load(path))
    idx = [int(i) for i in want["indices"]]
    bad = []
    for s, i in enumerate(idx):
        o = batch.oscillation(0, i)
        got = {"state": batch.state(i), "amps": o["amps"], "pers": o["pers"], "avg_peak": o["avg_peak"],
               "ncrit": o["ncrit"]}
        for k, v in got.items():
            w = want[("state_%d" if k == "state" else "a0_" + k + "_%d") % s]
            a, b = np.asarray(v, np.float64), np.asarray(w, np.float64)
            if a.shape != b.shape or not np.array_equal(np.isnan(a), np.isnan(b)) or \
                    not np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)]):
                bad.append("set %d %s" % (i, k))
    return {"fixture": PARITY_FIXTURE, "checked": True, "sets": idx, "bit_exact": not bad, "mismatches": bad,
            "what": "final state and mh1 oscillation amplitudes, periods, mean peaks and critical-point counts of "
                    "these sets after the timed run, against DENSE's own outputs"}


def cpu_sample(kind_pref="reference", num_sets=8, minutes=300.0, seed=7):
    """DENSE (or the oracle port) on the host, one core, a bounded sample:
    `num_sets` sets of the workload for `minutes` simulated minutes."""
    from dense_b200 import workloads
    from dense_b200.tissue import default_graph
    from oracle.pyoracle import load_oracle, load_ref
    lib = load_ref("her_model_2014") if kind_pref == "reference" else None
    kind = "reference"
    if lib is None:
        lib, kind = load_oracle("her_model_2014"), "port"
    P = workloads.log_uniform_params(num_sets, seed=seed)
    off, ids = default_graph(200, 4)
    mh1 = workloads.her_species("mh1")
    steps = 0
    t0 = time.perf_counter()
    for i in range(num_sets):
        sim = lib.create(off, ids, np.tile(P[i], (200, 1)), P[i], None, 0.01)
        sim.add_oscillation(mh1, 0, 200, 0.0, float("inf"), 4.0, 0.1)
        chunks = sim.run(minutes, 0.1)
        steps += chunks * int(0.1 / 0.01) * 200
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "cell-steps/s", "cores": 1, "kind": kind,
            "sample": "%d sets x 200 cells x %g min (dt 0.01, Oscillation mh1 every 0.1 min) of the workload, "
                      "one host core, %.1f s" % (num_sets, minutes, dt)}


# Turing-Pattern cell-step: 4 species read and written (8 B each); the
# neighbour averages read rows of the same arrays, so they add no distinct
# bytes.
TURING_BYTES_PER_CELL_STEP = 64
MIXED_BYTES = {"her_model_2014": BYTES_PER_CELL_STEP, "turing": TURING_BYTES_PER_CELL_STEP}
MIXED_WORKLOAD = ("uneven mixed batch, one captured graph: %d sets, her_model_2014 (cells log-uniform 16..1024, "
                  "-w 4, delays U[5,20] min) or Turing-Pattern (N x N grid, N U[8,64], -w N) with probability 1/2, "
                  "horizons U[100,1200] min, every rate x exp(U(ln .5, ln 2)), dt 0.01 min, no analyses, "
                  "autotuned schedules")


def mixed_cpu_sample(groups, minutes=60.0, per_model=4):
    """DENSE's own CPU path (oracle/_ref) on `per_model` sets of each model
    of the mixed batch, `minutes` each, one host core."""
    from oracle.pyoracle import load_oracle, load_ref
    kinds, steps = set(), 0
    t0 = time.perf_counter()
    for m, sets in groups.items():
        lib = load_ref(m)
        kind = "reference"
        if lib is None:
            lib, kind = load_oracle(m), "port"
        kinds.add(kind)
        for ps in sets[:per_model]:
            cp = np.tile(ps.set_params, (ps.num_cells, 1))
            sim = lib.create(ps.nbr_offsets, ps.nbr_ids, cp, ps.set_params, ps.init_conc, 0.01)
            chunks = sim.run(min(minutes, ps.duration), 1.0)
            steps += chunks * 100 * ps.num_cells
    dt = time.perf_counter() - t0
    return {"value": steps / dt, "unit": "cell-steps/s", "cores": 1,
            "kind": "reference" if kinds == {"reference"} else "port",
            "sample": "the first %d sets of each model of the mixed batch, %g min each, one host core, %.1f s"
                      % (per_model, minutes, dt)}


def run_mixed(a):
    """The uneven mixed batch (her_model_2014 + Turing-Pattern) in one graph."""
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from dense_b200 import workloads
    from dense_b200.autotune import Autotuner
    from dense_b200.mixed import MixedBatch

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    num_sets = a.sets if a.sets != 4096 else 10000
    groups = workloads.mixed_sets(num_sets, seed=3 + rank)
    t0 = time.perf_counter()
    tuner = Autotuner(device=local)
    chosen = {m: tuner.tune(m, sets, 0.01) for m, sets in groups.items()}
    tune_s = time.perf_counter() - t0
    mb = MixedBatch(groups, 0.01, 1.0, device=local)
    info = mb.info()
    per_step = int(math.ceil(1200.0 / a.steps))  # chunks of 1 min
    stream = torch.cuda.Stream()
    for _ in range(a.warmup):
        mb.run(per_step, stream=stream)
    barrier()
    mb.reset()
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    clocks = Clocks(local)
    barrier()
    ev[0].record(stream)
    for k in range(a.steps):
        mb.run(per_step, stream=stream)
        ev[k + 1].record(stream)
    stream.synchronize()
    barrier()
    clk = clocks.stop()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(a.steps)]
    total_ms = ev[0].elapsed_time(ev[a.steps])
    done = mb.done_cell_steps(100)
    done_bytes = 0
    for m, b in mb.batches.items():
        chunks, _ = b.progress()
        done_bytes += MIXED_BYTES[m] * int(sum(int(chunks[i]) * 100 * s.num_cells for i, s in enumerate(b.sets)))
    status_bad = int(sum(int((b.status() != 0).sum()) for b in mb.batches.values()))
    t = torch.tensor([total_ms, done], dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t[:1], op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(t[1:], op=torch.distributed.ReduceOp.SUM)
    total_ms_max, all_done = float(t[0]), float(t[1])
    value = all_done / (total_ms_max / 1e3)
    mb.close()

    # e2e: the batch built from host arrays, the whole horizon, every final state to the host
    e2e_times, h2d, d2h = [], 0, 0
    for k in range(a.e2e_steps):
        barrier()
        t1 = time.perf_counter()
        m2 = MixedBatch(groups, 0.01, 1.0, device=local)
        for b in m2.batches.values():
            b.run(-1)
        res = [b.state(i) for b in m2.batches.values() for i in range(len(b.sets))]
        m2.close()
        barrier()
        e2e_times.append(time.perf_counter() - t1)
        if k == 0:
            h2d = sum(s.set_params.nbytes + s.nbr_offsets.nbytes + s.nbr_ids.nbytes for v in groups.values()
                      for s in v)
            d2h = sum(r.nbytes for r in res)
    # per rank the median of the e2e steps, then the slowest rank
    e2e_s = statistics.median(e2e_times) if e2e_times else float("nan")
    if world > 1:
        x = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(x[0])
    hbm, peak_src = peaks()
    achieved = done_bytes / (total_ms / 1e3) / 1e9
    cpu = mixed_cpu_sample(groups) if (rank == 0 and world == 1 and not a.no_cpu) else None
    if rank == 0:
        from dense_b200.engine import plan
        # one launch per kernel group of each engine (register kernel, one per memory-kernel CTA size)
        n_launch = sum(len(set(plan(m, b.sets, 0.01, 1.0)[1].tolist())) for m, b in mb.batches.items())
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": total_ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": MIXED_WORKLOAD % num_sets,
                       "sets": {m: len(v) for m, v in groups.items()},
                       "step": "one graph replay advancing every unfinished set %d min" % per_step,
                       "schedules": {m: {"%d,%d" % k: list(v) for k, v in c.items()} for m, c in chosen.items()},
                       "autotune_s": tune_s,
                       "l2": "inputs larger than L2 (%.0f MB of rings per GPU)" % (info["device_bytes"] / 1e6),
                       "parallelism": "sets sharded across %d GPU(s), no exchange" % world},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None,
                         "basis": "algorithmic bytes %d per her cell-step, %d per Turing cell-step; peak %s"
                                  % (BYTES_PER_CELL_STEP, TURING_BYTES_PER_CELL_STEP, peak_src)},
            "cpu_baseline": cpu,
            "e2e": {"value": world * info["total_cell_steps"] / e2e_s, "unit": "cell-steps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": a.e2e_steps,
                    "what": "MixedBatch from host arrays + full horizons + every final state to host"},
            "gpu_launches": a.steps * n_launch,
            "clocks": clk,
            "step_ms": {"min": min(step_ms), "max": max(step_ms)},
            "status_nonzero_sets": status_bad,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_turing(a):
    """Turing-Pattern sets of one N x N grid (`--grid`), template parameters,
    the model's initial concentrations, dt 0.01 min, no analyses: the wave
    kernel alone."""
    import torch
    import numpy as np
    from dense_b200 import engine as E, workloads
    from dense_b200.tissue import default_graph
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    N = a.grid
    sets_n = a.sets if a.sets != 4096 else 148 * 6
    p = workloads.template_params("turing")
    ic = np.array(workloads.templates()["turing"]["init_conc"])
    off, ids = default_graph(N * N, N)
    sets = [E.ParameterSet(off, ids, p, init_conc=ic, duration=a.minutes) for _ in range(sets_n)]
    b = E.Batch("turing", sets, 0.01, 1.0 if a.minutes >= 1.0 else a.minutes, (), device=local)
    total_chunks = int(math.ceil(a.minutes / (1.0 if a.minutes >= 1.0 else a.minutes)))
    per_step = int(math.ceil(total_chunks / a.steps))
    stream = torch.cuda.Stream()
    for _ in range(a.warmup):
        b.run(per_step, stream=stream.cuda_stream, graph=True)
    b.reset(stream=stream.cuda_stream)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    clocks = Clocks(local)
    ev[0].record(stream)
    for k in range(a.steps):
        b.run(per_step, stream=stream.cuda_stream, graph=True)
        ev[k + 1].record(stream)
    stream.synchronize()
    clk = clocks.stop()
    ms = ev[0].elapsed_time(ev[a.steps])
    chunks, _ = b.progress()
    spc = b.info()["total_cell_steps"] // max(1, total_chunks) // sets_n // (N * N)
    done = int(chunks.astype(np.int64).sum()) * spc * N * N
    value = done / (ms / 1e3)
    status = int((b.status() != 0).sum())
    b.close()
    # e2e: the public API from host arrays (create, the whole horizon, every
    # set's final state back to the host)
    e2e_s, h2d, d2h, e2e_cells = [], 0, 0, 0
    for _ in range(max(1, a.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eb = E.Batch("turing", sets, 0.01, 1.0 if a.minutes >= 1.0 else a.minutes, (), device=local)
        eb.run(-1)
        states = [eb.state(i) for i in range(len(sets))]
        eb.sync()
        e2e_s.append(time.perf_counter() - t0)
        e2e_cells = eb.info()["total_cell_steps"]
        eb.close()
        h2d = sum(x.set_params.nbytes + x.init_conc.nbytes + x.nbr_offsets.nbytes + x.nbr_ids.nbytes for x in sets)
        d2h = sum(st.nbytes for st in states)
    cpu = None
    if not a.no_cpu:
        from oracle.pyoracle import load_oracle, load_ref
        lib, kind = load_ref("turing"), "reference"
        if lib is None:
            lib, kind = load_oracle("turing"), "port"
        cpu_minutes = max(1.0, round(2.5e7 / (N * N * 100)))
        t0 = time.perf_counter()
        sim = lib.create(off, ids, np.tile(p, (N * N, 1)), p, ic, 0.01)
        chunks = sim.run(cpu_minutes, 1.0)
        secs = time.perf_counter() - t0
        cpu = {"value": chunks * 100 * N * N / secs, "unit": "cell-steps/s", "cores": 1, "kind": kind,
               "sample": "one set of the grid for %g min on one host core, %.1f s" % (cpu_minutes, secs)}
    hbm, peak_src = peaks()
    achieved = TURING_BYTES_PER_CELL_STEP * value / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "Turing-Pattern %d sets of a %dx%d grid (-c %d -w %d), template parameters, "
                                   "dt 0.01 min, %g min, no analyses" % (sets_n, N, N, N * N, N, a.minutes)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None, "basis": "%d algorithmic bytes per Turing cell-step; peak %s"
                                                   % (TURING_BYTES_PER_CELL_STEP, peak_src)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_cells / statistics.median(e2e_s), "unit": "cell-steps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": len(e2e_s),
                    "what": "Batch() from host arrays + the whole horizon + every set's final state to host"},
            "gpu_launches": a.steps, "clocks": clk,
            "status_nonzero_sets": status}), flush=True)


def run_single(a):
    """One her_model_2014 set: 200 cells on DENSE's default tissue (-c 200
    -w 4), every parameter of every cell x U(0.95, 1.05) (seeded), dt 0.01
    min, 600 min, Basic over every species and cell and Oscillation of mh1
    and ph1 every 0.1 min.  A timed step is the whole 600-minute run of the
    set (reset before it, outside its events); one set occupies one SM, so
    the step is bound by the latency of its 60,000 dependent Euler steps."""
    import torch
    from dense_b200 import engine as E, workloads
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    minutes = a.minutes if a.minutes != 1200.0 else 600.0
    ps = workloads.perturbed_set(cells=200, width=4, duration=minutes, seed=1)
    an = workloads.cfg1_analyses(200, 0.1)
    b = E.Batch("her_model_2014", [ps], 0.01, 0.1, an, device=local)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    for _ in range(a.warmup):
        b.reset(stream=sptr)
        b.run(-1, stream=sptr)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    clocks = Clocks(local)
    for k in range(a.steps):
        b.reset(stream=sptr)
        ev[k][0].record(stream)
        b.run(-1, stream=sptr)
        ev[k][1].record(stream)
    stream.synchronize()
    clk = clocks.stop()
    step_ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    ms = sum(step_ms) / a.steps
    cell_steps = b.info()["total_cell_steps"]
    value = cell_steps / (ms / 1e3)
    status = int((b.status() != 0).sum())
    b.close()
    # e2e: the public API from host arrays: create (host->device), the run,
    # every analysis output of the set back to the host
    e2e_s, h2d, d2h = [], 0, 0
    for _ in range(max(1, a.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        eb = E.Batch("her_model_2014", [ps], 0.01, 0.1, an, device=local)
        eb.run(-1)
        basic, osc = eb.basic(0, 0), eb.oscillation(1, 0)
        eb.sync()
        e2e_s.append(time.perf_counter() - t0)
        eb.close()
        h2d = ps.set_params.nbytes + ps.cell_params.nbytes + ps.nbr_offsets.nbytes + ps.nbr_ids.nbytes
        d2h = sum(np.asarray(v).nbytes for v in list(basic.values()) + list(osc.values()))
    cpu = None
    if not a.no_cpu:
        from oracle.pyoracle import load_oracle, load_ref
        lib, kind = load_ref("her_model_2014"), "reference"
        if lib is None:
            lib, kind = load_oracle("her_model_2014"), "port"
        nsp = len(workloads.templates()["her_model_2014"]["species"])
        t0 = time.perf_counter()
        sim = lib.create(ps.nbr_offsets, ps.nbr_ids, ps.cell_params, ps.set_params, None, 0.01)
        sim.add_basic(list(range(nsp)), 0, 200, 0.0, float("inf"))
        sim.add_oscillation(workloads.her_species("mh1", "ph1"), 0, 200, 0.0, float("inf"), 4.0, 0.1)
        chunks = sim.run(minutes, 0.1)
        secs = time.perf_counter() - t0
        cpu = {"value": chunks * 10 * 200 / secs, "unit": "cell-steps/s", "cores": 1, "kind": kind,
               "sample": "the whole workload (one set, %g min) on one host core, %.1f s" % (minutes, secs)}
    hbm, peak_src = peaks()
    achieved = BYTES_PER_CELL_STEP * value / 1e9
    if rank == 0:
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": 1, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "her_model_2014, one set, 200 cells (-c 200 -w 4), every parameter of every cell "
                                   "x U(0.95, 1.05), dt 0.01 min, %g min, Basic (all species and cells) + "
                                   "Oscillation (mh1, ph1) every 0.1 min" % minutes,
                       "step": "the whole run of the set", "l2": "one set: state and history fit in L2"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                         "traffic": None,
                         "basis": "%d algorithmic bytes per cell-step; one set runs on one SM, so the step is "
                                  "latency-bound and far from either roofline; peak %s"
                                  % (BYTES_PER_CELL_STEP, peak_src)},
            "cpu_baseline": cpu,
            "e2e": {"value": cell_steps / statistics.median(e2e_s), "unit": "cell-steps/s",
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h), "steps": len(e2e_s),
                    "what": "Batch() from host arrays + the run + every analysis output to host"},
            "gpu_launches": a.steps, "clocks": clk,
            "step_ms": {"min": min(step_ms), "max": max(step_ms)},
            "status_nonzero_sets": status}), flush=True)


def _ref_worker(args):
    seed, minutes = args
    r = cpu_sample("reference", num_sets=1, minutes=minutes, seed=seed)
    return r["value"], r["kind"]


def run_reference(a):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    cores = len(os.sched_getaffinity(0))
    ctx = mp.get_context("spawn")
    minutes = 60.0
    with ctx.Pool(cores) as pool:
        for w in range(a.warmup):
            pool.map(_ref_worker, [(100 + w * cores + i, 10.0) for i in range(cores)])
        vals, kinds = [], set()
        t0 = time.perf_counter()
        for k in range(a.steps):
            out = pool.map(_ref_worker, [(1000 + k * cores + i, minutes) for i in range(cores)])
            kinds.update(x[1] for x in out)
        elapsed = time.perf_counter() - t0
    cell_steps = a.steps * cores * 200 * int(round(minutes / 0.1)) * 10
    value = cell_steps / elapsed
    kind = "reference" if kinds == {"reference"} else "port"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": elapsed / a.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": batch_workload(a.sets, a.minutes, True),  # the sample runs Oscillation
                       "sample_per_step": "%d sets x %g min of it, one set per core" % (cores, minutes)},
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": kind,
                             "sample": "%d host processes, each DENSE on one set of 200 cells for %g min per step"
                                       % (cores, minutes)},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--sets", type=int, default=4096)
    ap.add_argument("--minutes", type=float, default=1200.0)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--analyses", default="oscillation", choices=["oscillation", "none"],
                    help="the workload's analyses: Oscillation(mh1) every 0.1 min, or none")
    ap.add_argument("--workload", default="batch", choices=["batch", "mixed", "turing", "single"],
                    help="batch: 4096 her_model_2014 sets of 200 cells; mixed: the uneven her + Turing batch "
                         "(10000 sets unless --sets is given); turing: sets of one Turing grid (--grid); "
                         "single: one perturbed her_model_2014 set of 200 cells, 600 min, Basic + Oscillation")
    ap.add_argument("--grid", type=int, default=64, help="turing workload: grid side N")
    a = ap.parse_args()
    if a.impl == "reference":
        return run_reference(a)
    if a.workload == "mixed":
        return run_mixed(a)
    if a.workload == "turing":
        return run_turing(a)
    if a.workload == "single":
        return run_single(a)

    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from dense_b200 import engine as E

    precision = E.FP64 if a.precision == "fp64" else E.FP32_KAHAN
    sets, analyses = build_workload(a.sets, a.minutes, seed=2 + rank)
    if a.analyses == "none":
        analyses = []
    batch = E.Batch("her_model_2014", sets, 0.01, 0.1, analyses, precision=precision, device=local)
    info = batch.info()
    total_chunks = int(math.ceil(a.minutes / 0.1))
    per_step = int(math.ceil(total_chunks / a.steps))
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    for _ in range(a.warmup):
        batch.run(per_step, stream=sptr, graph=True)
    barrier()
    batch.reset(stream=sptr)
    barrier()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps + 1)]
    clocks = Clocks(local)
    barrier()
    ev[0].record(stream)
    for k in range(a.steps):
        batch.run(per_step, stream=sptr, graph=True)
        ev[k + 1].record(stream)
    stream.synchronize()
    barrier()
    clk = clocks.stop()
    step_ms = [ev[k].elapsed_time(ev[k + 1]) for k in range(a.steps)]
    total_ms = ev[0].elapsed_time(ev[a.steps])
    chunks, _ = batch.progress()
    status = batch.status()
    done_cell_steps = int(sum(int(chunks[i]) * 10 * sets[i].num_cells for i in range(len(sets))))
    # the timed run's results against DENSE's own on the workload's sets
    # it holds (the default workload on rank 0 only)
    parity = None
    if (rank == 0 and a.sets == 4096 and a.minutes == 1200.0 and analyses and precision == E.FP64):
        parity = batch_parity(batch)
    t = torch.tensor([total_ms, done_cell_steps], dtype=torch.float64, device="cuda")
    if world > 1:
        tm = t.clone()
        torch.distributed.all_reduce(tm[:1], op=torch.distributed.ReduceOp.MAX)
        torch.distributed.all_reduce(tm[1:], op=torch.distributed.ReduceOp.SUM)
        t = tm
    total_ms_max, all_cell_steps = float(t[0]), float(t[1])
    value = all_cell_steps / (total_ms_max / 1e3)
    per_launch_cell_steps = done_cell_steps / a.steps
    avg_launch_s = (total_ms / a.steps) / 1e3

    # ---- e2e through the public API, host buffers
    e2e_times = []
    h2d = d2h = 0
    e2e_clocks = Clocks(local)
    for k in range(a.e2e_steps):
        barrier()
        t0 = time.perf_counter()
        b = E.Batch("her_model_2014", sets, 0.01, 0.1, analyses, precision=precision, device=local)
        b.run(-1)
        if analyses:
            res = b.oscillation_all(0)          # every set's amplitudes and periods
        else:
            res = [b.state(i) for i in range(len(sets))]
        b.close()
        barrier()
        e2e_times.append(time.perf_counter() - t0)
        if k == 0:
            # parameters (one row per set, or per-cell rows), neighbour lists
            h2d = sum(s.set_params.nbytes + (s.cell_params.nbytes if s.cell_params is not None else 0) +
                      s.nbr_offsets.nbytes + s.nbr_ids.nbytes for s in sets)
            d2h = sum(r.nbytes for r in res)
    e2e_clk = e2e_clocks.stop()
    # per rank the median of the e2e steps, then the slowest rank
    e2e_s = statistics.median(e2e_times) if e2e_times else float("nan")
    if world > 1:
        x = torch.tensor([e2e_s], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(x, op=torch.distributed.ReduceOp.MAX)
        e2e_s = float(x[0])
    e2e_value = world * info["total_cell_steps"] / e2e_s

    hbm, peak_src = peaks()
    achieved_gbs = BYTES_PER_CELL_STEP * per_launch_cell_steps / avg_launch_s / 1e9
    # DRAM traffic of one launch, scaled from an ncu capture of a smaller
    # launch of the same kernel and workload shape (296 sets x 200 cells x
    # 1000 steps: dram__bytes_read.sum + dram__bytes_write.sum = 0.973 GB,
    # 16.4 B per cell-step, cold caches); FP64 with Oscillation only
    traffic = None
    if precision == E.FP64 and analyses:
        traffic = DRAM_BYTES_PER_CELL_STEP * per_launch_cell_steps

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu:
        cpu = cpu_sample()

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": total_ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if precision == E.FP64 else "f32+kahan", "data": "synthetic",
            "config": {"workload": batch_workload(a.sets, a.minutes, bool(analyses)),
                       "sets_per_gpu": a.sets, "step": "one launch advancing every set %d chunks (%g min)"
                       % (per_step, per_step * 0.1), "l2": "inputs larger than L2 (history rings + "
                       "windows %.0f MB per GPU)" % (info["device_bytes"] / 1e6),
                       "parallelism": "sets sharded across %d GPU(s), no exchange" % world},
            "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm, "unit": "GB/s",
                         "frac": achieved_gbs / hbm, "traffic": traffic,
                         "basis": "%d algorithmic bytes per cell-step (state read+write, delayed reads); peak "
                                  "%s" % (BYTES_PER_CELL_STEP, peak_src),
                         "fp64_flops_per_s": FLOPS_PER_CELL_STEP * per_launch_cell_steps / avg_launch_s},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "steps": a.e2e_steps,
                    "step_s": [round(x, 4) for x in e2e_times], "clocks": e2e_clk,
                    "what": "Batch() from host arrays + full horizon + every set's oscillation amplitudes and "
                            "periods to host; median of the steps"},
            "gpu_launches": a.steps,
            "clocks": clk,
            "step_ms": {"min": min(step_ms), "max": max(step_ms)},
            "status_nonzero_sets": int((status != 0).sum()),
            "parity": parity,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
