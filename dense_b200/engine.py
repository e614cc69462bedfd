"""Python host API over the engine's C ABI (include/dense_b200.h).

The objects mirror DENSE's own vocabulary: a batch of parameter sets (one
DENSE ``Deterministic_Simulation`` each), run by ``run_simulation``'s chunk
loop with ``BasicAnalysis``, ``OscillationAnalysis`` and
``ConcentrationCheck`` attached.  Every call goes through the CUDA library
of the model; there is no CPU path, and a missing library is an error.
"""

import ctypes as C
import os
import threading

import numpy as np

from . import build as _build

FP64 = 0
FP32_KAHAN = 1

BASIC = 1
OSCILLATION = 2
CONCCHECK = 3
TRAJECTORY = 4

SET_DROPPED = 1
SET_NAN_PARAM = 2
SET_UNSTAGED_LAG = 4
SET_BAD_DELAY = 8
SET_ORDERED_READS = 16
SCHEDULE_AUTO = 0
SCHEDULE_MEMORY = 1
SCHEDULE_GLOBAL = 2
SCHEDULE_SHARED_NEIGHBOUR = 3
SCHEDULE_WAVE_GLOBAL = 4
SCHEDULE_SHARED_ROWS = 5
SCHEDULE_REGISTER = 6

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class _ModelInfo(C.Structure):
    _fields_ = [("num_species", C.c_int), ("num_reactions", C.c_int), ("num_delay_reactions", C.c_int),
                ("num_critical_species", C.c_int), ("num_params", C.c_int)]


class _SetDesc(C.Structure):
    _fields_ = [("num_cells", C.c_int), ("nbr_offsets", _I), ("nbr_ids", _I), ("set_params", _D),
                ("cell_params", _D), ("init_conc", _D), ("perturb", _D), ("duration", C.c_double),
                ("schedule", C.c_int), ("mem_block", C.c_int)]


class _AnalysisDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("num_species", C.c_int), ("species", _I), ("cell_start", C.c_int),
                ("cell_end", C.c_int), ("time_start", C.c_double), ("time_end", C.c_double),
                ("win_range", C.c_double), ("anlys_intvl", C.c_double), ("lower", C.c_double),
                ("upper", C.c_double)]


class _RunDesc(C.Structure):
    _fields_ = [("precision", C.c_int), ("step_size", C.c_double), ("analysis_interval", C.c_double),
                ("num_analyses", C.c_int), ("analyses", C.POINTER(_AnalysisDesc)), ("device", C.c_int)]


_FUNCS = {
    "dense_model_get_info": (C.c_int, [C.POINTER(_ModelInfo)]),
    "dense_model_specie_name": (C.c_char_p, [C.c_int]),
    "dense_model_reaction_name": (C.c_char_p, [C.c_int]),
    "dense_model_delay_reaction_name": (C.c_char_p, [C.c_int]),
    "dense_model_critical_specie_name": (C.c_char_p, [C.c_int]),
    "dense_last_error": (C.c_char_p, []),
    "dense_engine_create": (C.c_int, [C.POINTER(_RunDesc), C.c_int, C.POINTER(_SetDesc), C.POINTER(C.c_void_p)]),
    "dense_engine_plan": (C.c_int, [C.POINTER(_RunDesc), C.c_int, C.POINTER(_SetDesc), C.POINTER(C.c_int64), _I,
                                    _I]),
    "dense_engine_run": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dense_engine_read_oscillation_all": (C.c_int, [C.c_void_p, C.c_int, _D, _D]),
    "dense_engine_copy_trajectory": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_int, _I, C.c_void_p]),
    "dense_engine_trajectory_capacity": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "dense_graph_capture": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int, C.c_int,
                                      C.POINTER(C.c_void_p)]),
    "dense_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dense_graph_destroy": (C.c_int, [C.c_void_p]),
    "dense_engine_run_graph": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "dense_engine_sync": (C.c_int, [C.c_void_p]),
    "dense_engine_reset": (C.c_int, [C.c_void_p, C.c_void_p]),
    "dense_engine_status": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32)]),
    "dense_engine_progress": (C.c_int, [C.c_void_p, C.POINTER(C.c_int32), _D]),
    "dense_engine_read_state": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "dense_engine_read_basic": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D, _D, _D, _D, _D, _I, _D]),
    "dense_engine_read_oscillation": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D, _D, _I, _I, _D]),
    "dense_engine_read_trajectory": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _D, _D, C.c_int, _I]),
    "dense_engine_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), _I]),
    "dense_engine_ring_info": (C.c_int, [C.c_void_p, C.c_int, _I, _I]),
    "dense_engine_analyze_samples": (C.c_int, [C.c_void_p, C.c_int, _D, C.c_int, C.c_double]),
    "dense_engine_checkpoint_size": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64)]),
    "dense_engine_checkpoint": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "dense_engine_restore": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64]),
    "dense_engine_destroy": (C.c_int, [C.c_void_p]),
}

_libs = {}
_lock = threading.Lock()


class DenseError(RuntimeError):
    pass


class ModelLibrary:
    """The engine library of one DENSE model."""

    def __init__(self, path):
        self.path = path
        self.lib = C.CDLL(path)
        for name, (res, args) in _FUNCS.items():
            f = getattr(self.lib, name)
            f.restype = res
            f.argtypes = args
        info = _ModelInfo()
        self._check(self.lib.dense_model_get_info(C.byref(info)))
        self.num_species = info.num_species
        self.num_reactions = info.num_reactions
        self.num_delay_reactions = info.num_delay_reactions
        self.num_critical_species = info.num_critical_species
        self.num_params = info.num_params
        self.species = [self.lib.dense_model_specie_name(i).decode() for i in range(self.num_species)]
        self.reactions = [self.lib.dense_model_reaction_name(i).decode() for i in range(self.num_reactions)]
        self.delay_reactions = [self.lib.dense_model_delay_reaction_name(i).decode()
                                for i in range(self.num_delay_reactions)]
        self.critical_species = [self.lib.dense_model_critical_specie_name(i).decode()
                                 for i in range(self.num_critical_species)]

    def _check(self, rc):
        if rc != 0:
            raise DenseError("dense_b200 error %d: %s" % (rc, self.lib.dense_last_error().decode()))

    def species_ids(self, names):
        if isinstance(names, str):
            names = [x.strip() for x in names.split(",") if x.strip()]
        return [self.species.index(n) if isinstance(n, str) else int(n) for n in names]


def load(model):
    """Load (building first if needed) the engine library of `model`."""
    with _lock:
        if model not in _libs:
            path = _build.build_model(model)
            if not os.path.exists(path):
                raise DenseError("engine library for %s missing" % model)
            _libs[model] = ModelLibrary(path)
        return _libs[model]


class ParameterSet:
    """One DENSE simulation: tissue, parameters, initial state, horizon."""

    def __init__(self, nbr_offsets, nbr_ids, set_params, cell_params=None, init_conc=None, perturb=None,
                 duration=0.0, schedule=0, mem_block=0):
        self.nbr_offsets = np.ascontiguousarray(nbr_offsets, np.int32)
        self.nbr_ids = np.ascontiguousarray(nbr_ids, np.int32)
        self.num_cells = len(self.nbr_offsets) - 1
        self.set_params = np.ascontiguousarray(set_params, np.float64)
        self.cell_params = None if cell_params is None else np.ascontiguousarray(cell_params, np.float64)
        self.init_conc = None if init_conc is None else np.ascontiguousarray(init_conc, np.float64)
        self.perturb = None if perturb is None else np.ascontiguousarray(perturb, np.float64)
        self.duration = float(duration)
        # schedule hints (SCHEDULE_*, memory-kernel CTA size); results do not depend on them
        self.schedule = int(schedule)
        self.mem_block = int(mem_block)


class Analysis:
    """One analysis entry (an <anlys> element of DENSE's analyses.xml)."""

    def __init__(self, kind, species=(), cell_start=0, cell_end=0, time_start=0.0, time_end=float("inf"),
                 win_range=0.0, anlys_intvl=0.0, lower=0.0, upper=0.0):
        self.kind = kind
        self.species = list(species)
        self.cell_start, self.cell_end = int(cell_start), int(cell_end)
        self.time_start, self.time_end = float(time_start), float(time_end)
        self.win_range, self.anlys_intvl = float(win_range), float(anlys_intvl)
        self.lower, self.upper = float(lower), float(upper)

    @staticmethod
    def basic(species, cell_start, cell_end, time_start=0.0, time_end=float("inf")):
        return Analysis(BASIC, species, cell_start, cell_end, time_start, time_end)

    @staticmethod
    def oscillation(species, cell_start, cell_end, time_start, time_end, win_range, anlys_intvl):
        return Analysis(OSCILLATION, species, cell_start, cell_end, time_start, time_end, win_range, anlys_intvl)

    @staticmethod
    def conccheck(species, cell_start, cell_end, lower, upper, time_start=0.0, time_end=float("inf")):
        return Analysis(CONCCHECK, species, cell_start, cell_end, time_start, time_end, lower=lower, upper=upper)

    @staticmethod
    def trajectory(species, cell_start, cell_end, time_start=0.0, time_end=float("inf")):
        """Every sample of the observed species (csvw_sim's data export)."""
        return Analysis(TRAJECTORY, species, cell_start, cell_end, time_start, time_end)


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


def _describe(L, sets, analyses, step_size, analysis_interval, precision, device):
    """C descriptors of a batch: (run desc, set desc array, arrays to keep alive)."""
    keep = []
    cset = (_SetDesc * len(sets))()
    for i, s in enumerate(sets):
        if s.cell_params is not None and s.cell_params.size != s.num_cells * L.num_params:
            raise DenseError("cell_params must be [num_cells][num_params]")
        if s.set_params.size != L.num_params:
            raise DenseError("set_params must have %d values" % L.num_params)
        cset[i].num_cells = s.num_cells
        cset[i].nbr_offsets = _ip(s.nbr_offsets)
        cset[i].nbr_ids = _ip(s.nbr_ids)
        cset[i].set_params = _dp(s.set_params)
        cset[i].cell_params = _dp(s.cell_params)
        cset[i].init_conc = _dp(s.init_conc)
        cset[i].perturb = _dp(s.perturb)
        cset[i].duration = s.duration
        cset[i].schedule = s.schedule
        cset[i].mem_block = s.mem_block
    can = (_AnalysisDesc * max(1, len(analyses)))()
    for i, a in enumerate(analyses):
        sp = np.ascontiguousarray(L.species_ids(a.species), np.int32)
        keep.append(sp)
        can[i].kind = a.kind
        can[i].num_species = len(sp)
        can[i].species = _ip(sp) if len(sp) else None
        can[i].cell_start, can[i].cell_end = a.cell_start, a.cell_end
        can[i].time_start, can[i].time_end = a.time_start, a.time_end
        can[i].win_range, can[i].anlys_intvl = a.win_range, a.anlys_intvl
        can[i].lower, can[i].upper = a.lower, a.upper
    run = _RunDesc(precision, float(step_size), float(analysis_interval), len(analyses), can, device)
    return run, cset, keep


def plan(model, sets, step_size, analysis_interval, analyses=(), precision=FP64):
    """Per-set device bytes, kernel (0 = register kernel, else the
    memory-state kernel's CTA size) and dependency levels per step (1 unless
    the set has ordered neighbour reads) that a Batch of these sets would
    use; needs no GPU."""
    L = load(model) if isinstance(model, str) else model
    sets = list(sets)
    run, cset, keep = _describe(L, sets, list(analyses), step_size, analysis_interval, precision, 0)
    nbytes = np.zeros(len(sets), np.int64)
    kernel = np.zeros(len(sets), np.int32)
    levels = np.zeros(len(sets), np.int32)
    L._check(L.lib.dense_engine_plan(C.byref(run), len(sets), cset, nbytes.ctypes.data_as(C.POINTER(C.c_int64)),
                                     _ip(kernel), _ip(levels)))
    return nbytes, kernel, levels


class Batch:
    """A batch of parameter sets staged on one GPU (dense_engine)."""

    def __init__(self, model, sets, step_size, analysis_interval, analyses=(), precision=FP64, device=0):
        self.L = load(model) if isinstance(model, str) else model
        self.sets = list(sets)
        self.analyses = list(analyses)
        self.precision = precision
        self.device = device
        L = self.L
        run, cset, self._keep = _describe(L, self.sets, self.analyses, step_size, analysis_interval, precision,
                                          device)
        h = C.c_void_p()
        L._check(L.lib.dense_engine_create(C.byref(run), len(self.sets), cset, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.lib.dense_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, num_chunks=-1, stream=None, graph=False):
        f = self.L.lib.dense_engine_run_graph if graph else self.L.lib.dense_engine_run
        self.L._check(f(self.h, int(num_chunks), stream))

    def sync(self):
        self.L._check(self.L.lib.dense_engine_sync(self.h))

    def reset(self, stream=None):
        self.L._check(self.L.lib.dense_engine_reset(self.h, stream))

    def status(self):
        out = np.zeros(len(self.sets), np.int32)
        self.L._check(self.L.lib.dense_engine_status(self.h, out.ctypes.data_as(C.POINTER(C.c_int32))))
        return out

    def progress(self):
        ch = np.zeros(len(self.sets), np.int32)
        age = np.zeros(len(self.sets), np.float64)
        self.L._check(self.L.lib.dense_engine_progress(self.h, ch.ctypes.data_as(C.POINTER(C.c_int32)), _dp(age)))
        return ch, age

    def state(self, set_index):
        n = self.sets[set_index].num_cells
        out = np.zeros((self.L.num_species, n), np.float64)
        self.L._check(self.L.lib.dense_engine_read_state(self.h, set_index, _dp(out)))
        return out

    def basic(self, analysis, set_index):
        a = self.analyses[analysis]
        k, m = len(a.species), a.cell_end - a.cell_start
        mins, sums, maxs = (np.zeros(k) for _ in range(3))
        cmins, csums, cmaxs = (np.zeros((m, k)) for _ in range(3))
        samples = C.c_int()
        time = C.c_double()
        self.L._check(self.L.lib.dense_engine_read_basic(self.h, analysis, set_index, _dp(mins), _dp(sums),
                                                         _dp(maxs), _dp(cmins), _dp(csums), _dp(cmaxs),
                                                         C.byref(samples), C.byref(time)))
        return dict(mins=mins, sums=sums, maxs=maxs, cell_mins=cmins, cell_sums=csums, cell_maxs=cmaxs,
                    samples=samples.value, time=time.value)

    def oscillation(self, analysis, set_index):
        a = self.analyses[analysis]
        k, m = len(a.species), a.cell_end - a.cell_start
        amps, pers, peaks = (np.zeros((k, m)) for _ in range(3))
        ncrit = np.zeros((k, m), np.int32)
        samples = C.c_int()
        time = C.c_double()
        self.L._check(self.L.lib.dense_engine_read_oscillation(self.h, analysis, set_index, _dp(amps), _dp(pers),
                                                               _dp(peaks), _ip(ncrit), C.byref(samples),
                                                               C.byref(time)))
        return dict(amps=amps, pers=pers, avg_peak=peaks, ncrit=ncrit, samples=samples.value, time=time.value)

    def trajectory(self, analysis, set_index):
        """Sample times [k] and values [k][species][cells] recorded so far."""
        a = self.analyses[analysis]
        n, m = len(a.species), a.cell_end - a.cell_start
        k = C.c_int()
        self.L._check(self.L.lib.dense_engine_read_trajectory(self.h, analysis, set_index, None, None, 0, C.byref(k)))
        times = np.zeros(k.value)
        vals = np.zeros((k.value, n, m))
        self.L._check(self.L.lib.dense_engine_read_trajectory(self.h, analysis, set_index, _dp(times), _dp(vals),
                                                              k.value, C.byref(k)))
        return times, vals

    def oscillation_all(self, analysis):
        """Every set's amplitudes and periods, [sets][species][cells]."""
        a = self.analyses[analysis]
        shape = (len(self.sets), len(a.species), a.cell_end - a.cell_start)
        amps, pers = np.zeros(shape), np.zeros(shape)
        self.L._check(self.L.lib.dense_engine_read_oscillation_all(self.h, analysis, _dp(amps), _dp(pers)))
        return amps, pers

    def trajectory_device(self, analysis):
        """Every set's recorded trajectory as a CUDA tensor [sets][capacity]
        [species][cells] (float64, device to device) and each set's sample
        count (numpy)."""
        import torch
        a = self.analyses[analysis]
        cap = C.c_int()
        self.L._check(self.L.lib.dense_engine_trajectory_capacity(self.h, analysis, C.byref(cap)))
        out = torch.empty((len(self.sets), cap.value, len(a.species), a.cell_end - a.cell_start),
                          dtype=torch.float64, device="cuda:%d" % self.device)
        cnt = np.zeros(len(self.sets), np.int32)
        self.L._check(self.L.lib.dense_engine_copy_trajectory(self.h, analysis, C.c_void_p(out.data_ptr()), 1,
                                                              _ip(cnt), None))
        return out, cnt

    def info(self):
        cs = C.c_int64()
        nb = C.c_int64()
        bt = C.c_int()
        self.L._check(self.L.lib.dense_engine_info(self.h, C.byref(cs), C.byref(nb), C.byref(bt)))
        return dict(total_cell_steps=cs.value, device_bytes=nb.value, block_threads=bt.value)

    def analyze_samples(self, set_index, samples, time_start=0.0):
        """Runs the set's analyses over imported samples [k][species][cells]
        (simulation -i) instead of simulating; read the results as after a
        run."""
        x = np.ascontiguousarray(samples, np.float64)
        k = x.shape[0] if x.ndim == 3 else 0
        self.L._check(self.L.lib.dense_engine_analyze_samples(self.h, set_index, _dp(x), k, float(time_start)))

    def checkpoint(self):
        """The batch's whole run state so far, as bytes (waits for the
        engine's work): restore() on a Batch built from the same inputs --
        in this process or another -- continues from exactly this point."""
        n = C.c_int64()
        self.L._check(self.L.lib.dense_engine_checkpoint_size(self.h, C.byref(n)))
        buf = np.empty(n.value, np.uint8)
        self.L._check(self.L.lib.dense_engine_checkpoint(self.h, buf.ctypes.data_as(C.c_void_p), n.value))
        return buf.tobytes()

    def restore(self, snapshot):
        """Puts a checkpoint() of a batch with the same layout back."""
        buf = np.frombuffer(snapshot, np.uint8)
        self.L._check(self.L.lib.dense_engine_restore(self.h, buf.ctypes.data_as(C.c_void_p), buf.size))

    def ring_info(self, set_index):
        S = np.zeros(self.L.num_species, np.int32)
        D = np.zeros(self.L.num_species, np.int32)
        self.L._check(self.L.lib.dense_engine_ring_info(self.h, set_index, _ip(S), _ip(D)))
        return S, D
