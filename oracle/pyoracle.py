"""ctypes wrapper over the oracle C interface (test infrastructure only).

The same interface is exported by the CPU restatement
(``oracle/_lib/libdense_oracle_<model>.so``) and by the DENSE harness
(``oracle/_ref/libdense_ref_<model>.so``), so one wrapper drives both.
"""

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_D = C.POINTER(C.c_double)
_I = C.POINTER(C.c_int)


class _Info(C.Structure):
    _fields_ = [("num_species", C.c_int), ("num_reactions", C.c_int),
                ("num_delay_reactions", C.c_int), ("num_critical_species", C.c_int),
                ("num_params", C.c_int)]


def _dp(a):
    return None if a is None else a.ctypes.data_as(_D)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_I)


class OracleLib:
    """One loaded oracle library (restatement or DENSE harness) for one model."""

    def __init__(self, path):
        self.path = path
        lib = C.CDLL(path)
        self.lib = lib
        lib.oracle_model_info_get.argtypes = [C.POINTER(_Info)]
        lib.oracle_specie_name.restype = C.c_char_p
        lib.oracle_specie_name.argtypes = [C.c_int]
        lib.oracle_reaction_name.restype = C.c_char_p
        lib.oracle_reaction_name.argtypes = [C.c_int]
        lib.oracle_default_graph.argtypes = [C.c_int, C.c_int, _I, _I]
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [C.c_int, _I, _I, _D, _D, _D, C.c_double, _D]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        lib.oracle_ring_sizes.argtypes = [C.c_void_p, _I, _D]
        lib.oracle_add_basic.argtypes = [C.c_void_p, C.c_int, _I, C.c_int, C.c_int, C.c_double, C.c_double]
        lib.oracle_add_oscillation.argtypes = [C.c_void_p, C.c_int, _I, C.c_int, C.c_int, C.c_double,
                                               C.c_double, C.c_double, C.c_double]
        lib.oracle_add_conccheck.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double,
                                             C.c_double, C.c_double, C.c_double]
        lib.oracle_steps.argtypes = [C.c_void_p, C.c_long]
        lib.oracle_replay.restype = C.c_long
        lib.oracle_replay.argtypes = [C.c_void_p, _D, C.c_long, C.c_double, C.c_double]
        lib.oracle_run.restype = C.c_long
        lib.oracle_run.argtypes = [C.c_void_p, C.c_double, C.c_double]
        lib.oracle_status.argtypes = [C.c_void_p]
        lib.oracle_age.restype = C.c_double
        lib.oracle_age.argtypes = [C.c_void_p]
        lib.oracle_get_state.argtypes = [C.c_void_p, _D]
        lib.oracle_get_history.argtypes = [C.c_void_p, C.c_int, _D]
        lib.oracle_get_basic.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _D, _D, _D, _I, _D]
        lib.oracle_get_oscillation.argtypes = [C.c_void_p, C.c_int, _D, _D, _D, _I, _I, _D]
        lib.oracle_get_crits.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, _D, _D, _I, C.c_int]
        info = _Info()
        lib.oracle_model_info_get(C.byref(info))
        self.num_species = info.num_species
        self.num_reactions = info.num_reactions
        self.num_delay_reactions = info.num_delay_reactions
        self.num_critical_species = info.num_critical_species
        self.num_params = info.num_params
        self.species = [lib.oracle_specie_name(i).decode() for i in range(self.num_species)]
        self.reactions = [lib.oracle_reaction_name(i).decode() for i in range(self.num_reactions)]

    def default_graph(self, cells, width):
        off = np.zeros(cells + 1, np.int32)
        idx = np.zeros(6 * cells, np.int32)
        n = self.lib.oracle_default_graph(cells, width, _ip(off), _ip(idx))
        if n < 0:
            raise RuntimeError("default_graph not provided by %s" % self.path)
        return off, idx[:n].copy()

    def create(self, off, idx, cell_params, set_params, init_conc, dt, pert=None):
        return OracleSim(self, off, idx, cell_params, set_params, init_conc, dt, pert)


class OracleSim:
    """One simulation (one parameter set) in an oracle library."""

    def __init__(self, lib, off, idx, cell_params, set_params, init_conc, dt, pert=None):
        self.L = lib
        self.cells = len(off) - 1
        self._keep = [np.ascontiguousarray(off, np.int32), np.ascontiguousarray(idx, np.int32),
                      np.ascontiguousarray(cell_params, np.float64).reshape(self.cells, lib.num_params),
                      np.ascontiguousarray(set_params, np.float64),
                      None if init_conc is None else np.ascontiguousarray(init_conc, np.float64),
                      None if pert is None else np.ascontiguousarray(pert, np.float64)]
        k = self._keep
        self.h = lib.lib.oracle_create(self.cells, _ip(k[0]), _ip(k[1]), _dp(k[2]), _dp(k[3]), _dp(k[4]),
                                       float(dt), _dp(k[5]))
        self.analyses = []

    def __del__(self):
        if getattr(self, "h", None):
            self.L.lib.oracle_destroy(self.h)
            self.h = None

    def ring_sizes(self):
        S = np.zeros(self.L.num_species, np.int32)
        md = np.zeros(self.L.num_species, np.float64)
        self.L.lib.oracle_ring_sizes(self.h, _ip(S), _dp(md))
        return S, md

    def add_basic(self, species, cell_start, cell_end, t0=0.0, t1=float("inf")):
        sp = np.ascontiguousarray(species, np.int32)
        i = self.L.lib.oracle_add_basic(self.h, len(sp), _ip(sp), cell_start, cell_end, t0, t1)
        self.analyses.append(("basic", len(sp), cell_end - cell_start))
        return i

    def add_oscillation(self, species, cell_start, cell_end, t0, t1, win_range, anlys_intvl):
        sp = np.ascontiguousarray(species, np.int32)
        i = self.L.lib.oracle_add_oscillation(self.h, len(sp), _ip(sp), cell_start, cell_end, t0, t1,
                                              win_range, anlys_intvl)
        self.analyses.append(("oscillation", len(sp), cell_end - cell_start))
        return i

    def add_conccheck(self, target, cell_start, cell_end, lo, hi, t0=0.0, t1=float("inf")):
        i = self.L.lib.oracle_add_conccheck(self.h, target, cell_start, cell_end, lo, hi, t0, t1)
        if i >= 0:
            self.analyses.append(("conccheck", 0, 0))
        return i

    def steps(self, n):
        self.L.lib.oracle_steps(self.h, int(n))

    def replay(self, samples, time_start, interval):
        """The analyses over imported samples [k][species][cells]."""
        x = np.ascontiguousarray(samples, np.float64)
        return self.L.lib.oracle_replay(self.h, _dp(x), x.shape[0], float(time_start), float(interval))

    def run(self, duration, interval):
        return self.L.lib.oracle_run(self.h, float(duration), float(interval))

    def status(self):
        return self.L.lib.oracle_status(self.h)

    def age(self):
        return self.L.lib.oracle_age(self.h)

    def state(self):
        out = np.zeros((self.L.num_species, self.cells), np.float64)
        self.L.lib.oracle_get_state(self.h, _dp(out))
        return out

    def history(self, sp):
        S, _ = self.ring_sizes()
        out = np.zeros((S[sp], self.cells), np.float64)
        self.L.lib.oracle_get_history(self.h, sp, _dp(out))
        return out

    def basic(self, idx):
        _, n, nc = self.analyses[idx]
        mins, sums, maxs = (np.zeros(n) for _ in range(3))
        cmins, csums, cmaxs = (np.zeros((nc, n)) for _ in range(3))
        samples = C.c_int()
        time = C.c_double()
        self.L.lib.oracle_get_basic(self.h, idx, _dp(mins), _dp(sums), _dp(maxs), _dp(cmins), _dp(csums),
                                    _dp(cmaxs), C.byref(samples), C.byref(time))
        return dict(mins=mins, sums=sums, maxs=maxs, cell_mins=cmins, cell_sums=csums, cell_maxs=cmaxs,
                    samples=samples.value, time=time.value)

    def oscillation(self, idx):
        _, n, nc = self.analyses[idx]
        amps, pers, peaks = (np.zeros((n, nc)) for _ in range(3))
        ncrit = np.zeros((n, nc), np.int32)
        samples = C.c_int()
        time = C.c_double()
        self.L.lib.oracle_get_oscillation(self.h, idx, _dp(amps), _dp(pers), _dp(peaks), _ip(ncrit),
                                          C.byref(samples), C.byref(time))
        return dict(amps=amps, pers=pers, avg_peak=peaks, ncrit=ncrit, samples=samples.value,
                    time=time.value)

    def crits(self, idx, s, c, cap=100000):
        t = np.zeros(cap)
        conc = np.zeros(cap)
        pk = np.zeros(cap, np.int32)
        n = self.L.lib.oracle_get_crits(self.h, idx, s, c, _dp(t), _dp(conc), _ip(pk), cap)
        return t[:n].copy(), conc[:n].copy(), pk[:n].astype(bool)


def load_oracle(model):
    from oracle.build import build_oracle
    return OracleLib(build_oracle(model))


def load_ref(model):
    """DENSE itself, or None where its build is absent."""
    from oracle.build import ref_lib_path, build_ref
    p = ref_lib_path(model)
    if not os.path.exists(p):
        try:
            p = build_ref(model, cli=False)
        except Exception:
            return None
    return OracleLib(p) if p and os.path.exists(p) else None
