"""Schedule autotuner for uneven batches.

A set's results do not depend on how it is scheduled, only its speed does:
the register kernel (one thread per cell, the whole state in registers;
unordered sets of at most 256 cells) or the memory-state kernel with a CTA
of 32..256 threads (any set; cells beyond the CTA width loop, so the CTA
size is the cells-per-thread knob), or for sets with in-order neighbour
reads the wave kernel, whose CTA holds one thread group per time step in
flight (so there the CTA size also sets how many steps overlap).  History depth is not a knob: each
species' ring holds exactly the lags its reads need, rounded up to a power
of two.

The tuner buckets sets by model, dependency kind (ordered neighbour reads
or not) and cell count (powers of two), times every candidate schedule of
a bucket on a sample of its sets replicated to fill the GPU for a short
horizon, and stamps the fastest schedule on every set of the bucket
(ParameterSet.schedule / .mem_block).  Choices are cached per
(model, bucket, GPU name) in a JSON file when one is given.
"""

import copy
import json
import math
import os

import numpy as np

from . import engine as E

MEM_BLOCKS = (32, 64, 128, 256)


def bucket_of(s, levels):
    """(ordered, log2 cell-count bucket) of a set; levels is its number of
    dependency levels per step (more than 1: ordered neighbour reads)."""
    return (bool(levels > 1), int(math.ceil(math.log2(max(2, s.num_cells)))))


def candidates(ordered, cells_log2):
    """Schedules worth timing for a bucket: (schedule, mem_block) pairs.
    Ordered sets: the wave kernel with the engine's CTA (one thread group
    per step in flight) or one or two warps (fewer steps in flight, more
    sets per SM), only the neighbour-read species in shared memory, or
    every row in global memory; others: the register kernel (up to 256
    cells) or the memory kernel with a CTA no wider than the set."""
    if ordered:
        return [(E.SCHEDULE_MEMORY, 0), (E.SCHEDULE_MEMORY, 32), (E.SCHEDULE_MEMORY, 64),
                (E.SCHEDULE_SHARED_NEIGHBOUR, 0), (E.SCHEDULE_WAVE_GLOBAL, 0)]
    cells = 1 << cells_log2
    out = [(E.SCHEDULE_AUTO, 0)] if cells <= 256 else []
    out += [(E.SCHEDULE_MEMORY, b) for b in MEM_BLOCKS if b <= max(32, cells)]
    return out


def _with(s, schedule, mem_block, duration):
    t = copy.copy(s)
    t.schedule, t.mem_block, t.duration = schedule, mem_block, duration
    return t


def time_schedule(model, sample, schedule, mem_block, step_size, minutes=1.0, fill_cells=1 << 19,
                  device=0, repeats=2):
    """Cell-steps/s of `sample` (replicated to about `fill_cells` cells) run
    `minutes` under one schedule; CUDA events on a private stream."""
    import torch
    n = sum(s.num_cells for s in sample)
    reps = max(1, int(math.ceil(fill_cells / max(1, n))))
    sets = [_with(s, schedule, mem_block, minutes) for _ in range(reps) for s in sample]
    interval = minutes
    b = E.Batch(model, sets, step_size, interval, (), device=device)
    try:
        stream = torch.cuda.Stream(device=device)
        ptr = stream.cuda_stream
        b.run(-1, stream=ptr)  # warm-up (first launches set kernel attributes)
        best = float("inf")
        for _ in range(repeats):
            b.reset(stream=ptr)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            b.run(-1, stream=ptr)
            e1.record(stream)
            stream.synchronize()
            best = min(best, e0.elapsed_time(e1) / 1e3)
        return b.info()["total_cell_steps"] / best
    finally:
        b.close()


class Autotuner:
    """`timer(model, sample, schedule, mem_block, step_size, minutes,
    device=...)` gives a schedule's cell-steps/s (time_schedule by default);
    `gpu_name` keys the cache (the device's name by default)."""

    def __init__(self, cache_path=None, sample_sets=8, minutes=1.0, device=0, verbose=False, timer=None,
                 gpu_name=None):
        self.cache_path = cache_path
        self.sample_sets = sample_sets
        self.minutes = minutes
        self.device = device
        self.verbose = verbose
        self.timer = timer or time_schedule
        self.gpu_name = gpu_name
        self.cache = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)
        self.log = []

    def _key(self, model, bucket):
        if self.gpu_name is None:
            import torch
            self.gpu_name = torch.cuda.get_device_name(self.device)
        return "%s|%s|%d|%d" % (self.gpu_name, model, bucket[0], bucket[1])

    def tune(self, model, sets, step_size):
        """Stamp the fastest schedule of each bucket on `sets` (in place);
        returns {bucket: (schedule, mem_block)}."""
        _, _, levels = E.plan(model, sets, step_size, 1.0)
        groups = {}
        for i, s in enumerate(sets):
            if s.schedule != E.SCHEDULE_AUTO or s.mem_block:
                continue  # the caller chose already
            groups.setdefault(bucket_of(s, levels[i]), []).append(i)
        chosen = {}
        for bucket, idx in sorted(groups.items()):
            key = self._key(model, bucket)
            if key in self.cache:
                chosen[bucket] = tuple(self.cache[key])
            else:
                rng = np.random.Generator(np.random.PCG64(len(idx)))
                pick = rng.choice(idx, size=min(self.sample_sets, len(idx)), replace=False)
                sample = [sets[i] for i in pick]
                results = []
                cands = candidates(bucket[0], bucket[1])
                for cand in cands if len(cands) > 1 else []:
                    v = self.timer(model, sample, cand[0], cand[1], step_size, self.minutes, device=self.device)
                    results.append((v, cand))
                    self.log.append({"model": model, "bucket": bucket, "schedule": cand, "cell_steps_per_s": v})
                    if self.verbose:
                        print("autotune", model, bucket, cand, "%.3e" % v, flush=True)
                chosen[bucket] = max(results)[1] if results else cands[0]
                self.cache[key] = list(chosen[bucket])
            for i in idx:
                sets[i].schedule, sets[i].mem_block = chosen[bucket]
        if self.cache_path:
            with open(self.cache_path, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
        return chosen
