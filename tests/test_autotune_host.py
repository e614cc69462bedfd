"""The uneven mixed batch on the host: the schedule autotuner's logic
(dense_b200.autotune) with a fake timer in place of GPU timing -- buckets,
candidate schedules, stamping every set of a bucket with its fastest
schedule, leaving the caller's own choices alone, the per-GPU cache -- and
the workload generator (dense_b200.workloads.mixed_sets)."""

import json

from dense_b200 import engine as E, workloads
from dense_b200.autotune import MEM_BLOCKS, Autotuner, bucket_of, candidates


def test_bucket_of():
    s = workloads.perturbed_set(cells=200, width=4, duration=1.0)
    assert bucket_of(s, 1) == (False, 8)
    assert bucket_of(s, 7) == (True, 8)
    one = E.ParameterSet([0, 0], [], workloads.template_params(), duration=1.0)
    assert bucket_of(one, 1) == (False, 1)


def test_candidates():
    assert candidates(False, 4) == [(E.SCHEDULE_AUTO, 0), (E.SCHEDULE_MEMORY, 32)]
    assert candidates(False, 8) == [(E.SCHEDULE_AUTO, 0)] + [(E.SCHEDULE_MEMORY, b) for b in MEM_BLOCKS]
    assert candidates(False, 10) == [(E.SCHEDULE_MEMORY, b) for b in MEM_BLOCKS]  # past the register kernel
    ordered = candidates(True, 12)
    assert (E.SCHEDULE_WAVE_GLOBAL, 0) in ordered and (E.SCHEDULE_SHARED_NEIGHBOUR, 0) in ordered
    assert all(s != E.SCHEDULE_AUTO for s, _ in ordered)


class FakeTimer:
    """Scores a schedule by a fixed preference; records what it timed."""

    def __init__(self, best):
        self.best = best
        self.calls = []

    def __call__(self, model, sample, schedule, mem_block, step_size, minutes, device=0):
        self.calls.append((model, len(sample), schedule, mem_block))
        return 2.0 if (schedule, mem_block) in self.best else 1.0 + mem_block / 1e4


def test_tune_stamps_buckets_and_caches(tmp_path):
    groups = workloads.mixed_sets(40, seed=5)
    her, turing = groups["her_model_2014"], groups["turing"]
    her[0].schedule, her[0].mem_block = E.SCHEDULE_GLOBAL, 64  # the caller's own choice stays
    cache = str(tmp_path / "tune.json")
    best = {(E.SCHEDULE_MEMORY, 64), (E.SCHEDULE_WAVE_GLOBAL, 0)}
    timer = FakeTimer(best)
    tuner = Autotuner(cache_path=cache, sample_sets=2, timer=timer, gpu_name="fake-gpu")
    chosen_her = tuner.tune("her_model_2014", her, 0.01)
    chosen_turing = tuner.tune("turing", turing, 0.01)

    assert (her[0].schedule, her[0].mem_block) == (E.SCHEDULE_GLOBAL, 64)
    _, _, lv = E.plan("her_model_2014", her, 0.01, 1.0)
    for i, s in enumerate(her[1:], 1):
        b = bucket_of(s, lv[i])
        assert (s.schedule, s.mem_block) == chosen_her[b]
        cands = candidates(*b)
        if len(cands) == 1:
            assert chosen_her[b] == cands[0]
        elif (E.SCHEDULE_MEMORY, 64) in cands:
            assert chosen_her[b] == (E.SCHEDULE_MEMORY, 64)
    for b, c in chosen_turing.items():
        assert b[0] and c == (E.SCHEDULE_WAVE_GLOBAL, 0)  # every Turing grid has ordered reads
    assert all(s.schedule == E.SCHEDULE_WAVE_GLOBAL for s in turing)
    # samples are at most sample_sets sets; every multi-candidate bucket was timed
    assert all(n <= 2 for _, n, _, _ in timer.calls)

    saved = json.load(open(cache))
    assert all(k.startswith("fake-gpu|") for k in saved) and len(saved) == len(chosen_her) + len(chosen_turing)

    # a second tuner on the same cache times nothing and chooses the same
    again = workloads.mixed_sets(40, seed=5)
    timer2 = FakeTimer(set())
    t2 = Autotuner(cache_path=cache, sample_sets=2, timer=timer2, gpu_name="fake-gpu")
    assert t2.tune("turing", again["turing"], 0.01) == chosen_turing
    assert timer2.calls == []


def test_mixed_workload_matches_its_description():
    """The uneven mixed batch: her_model_2014 (cells 16..1024 in multiples
    of 4, width 4, delays U[5, 20] min) or Turing-Pattern (N x N, N in
    8..64, width N) with probability 1/2, horizons U[100, 1200] min, rates
    scaled within [1/2, 2]; the same seed gives the same batch."""
    import numpy as np
    L = E.load("her_model_2014")
    d0, d1 = L.num_reactions, L.num_reactions + L.num_delay_reactions
    g = workloads.mixed_sets(400, seed=3)
    her, tur = g["her_model_2014"], g["turing"]
    assert len(her) + len(tur) == 400 and 150 < len(her) < 250
    hp, tp = workloads.template_params("her_model_2014"), workloads.template_params("turing")
    for s in her:
        assert 16 <= s.num_cells <= 1024 and s.num_cells % 4 == 0
        assert 100.0 <= s.duration <= 1200.0
        assert ((s.set_params[d0:d1] >= 5.0) & (s.set_params[d0:d1] <= 20.0)).all()
        nz = hp[:d0] > 0
        r = s.set_params[:d0][nz] / hp[:d0][nz]
        assert (r >= 0.5 - 1e-12).all() and (r <= 2.0 + 1e-12).all()
    for s in tur:
        n = int(round(np.sqrt(s.num_cells)))
        assert n * n == s.num_cells and 8 <= n <= 64 and 100.0 <= s.duration <= 1200.0
        nz = tp > 0
        r = s.set_params[nz] / tp[nz]
        assert (r >= 0.5 - 1e-12).all() and (r <= 2.0 + 1e-12).all()
        assert s.init_conc is not None
    again = workloads.mixed_sets(400, seed=3)
    assert [s.num_cells for s in again["turing"]] == [s.num_cells for s in tur]
    assert all(np.array_equal(a.set_params, b.set_params) for a, b in zip(again["her_model_2014"], her))
