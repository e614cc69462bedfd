"""DENSE's CSV number reader (csvr::get_real, io/csvr.cpp:56-110).

Kept token for token, because parameter files are read through it:

* the stream is read with ``>>``, so all whitespace, newlines included, is
  skipped -- a value is emitted only when a ',' ends it, and the last value
  of a file without a trailing comma is dropped;
* '#' discards the rest of the line;
* any character other than digits, '.', ',', 'e', '-', '+' discards
  everything up to and including the next ',';
* a token is converted with strtold and then narrowed to double, so the
  same double rounding applies;
* a token strtold cannot consume entirely ends the read.
"""

import ctypes
import ctypes.util

_libc = ctypes.CDLL(ctypes.util.find_library("c") or None)
_libc.strtold.restype = ctypes.c_longdouble
_libc.strtold.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p)]

_ALLOWED = set("0123456789.,\ne-+")


def _strtold_to_double(token):
    buf = ctypes.create_string_buffer(token.encode())
    end = ctypes.c_char_p()
    v = _libc.strtold(buf, ctypes.byref(end))
    consumed = ctypes.cast(end, ctypes.c_void_p).value - ctypes.addressof(buf)
    return float(v), consumed == len(token.encode())


def read_reals(text):
    """All values csvr::get_next would return, in order."""
    out = []
    i, n = 0, len(text)
    tok = ""
    while i < n:
        c = text[i]
        i += 1
        if c.isspace():
            continue
        if c == "#":
            j = text.find("\n", i)
            i = n if j < 0 else j + 1
            tok = ""
            continue
        if c not in _ALLOWED:
            j = text.find(",", i)
            i = n if j < 0 else j + 1
            tok = ""
            continue
        if c != "," and c != "\n":
            tok += c
            continue
        if tok:
            v, ok = _strtold_to_double(tok)
            if not ok:
                return out
            out.append(v)
            tok = ""
    return out


def read_param_sets(text, num_params):
    """csvr::get_param_sets (io/csvr.cpp:25-34): consecutive groups of
    num_params values; a partial last group is an error, as in DENSE."""
    vals = read_reals(text)
    if len(vals) % num_params:
        raise ValueError("partial parameter set at the end of the file (%d values, %d per set)"
                         % (len(vals), num_params))
    return [vals[k:k + num_params] for k in range(0, len(vals), num_params)]


def read_init_conc(text, num_species):
    """conc_vector (Sim_Initializer.hpp:138-157): values in order, truncated
    or zero-padded to num_species."""
    vals = read_reals(text)[:num_species]
    return vals + [0.0] * (num_species - len(vals))


def _number(cell):
    v, ok = _strtold_to_double(cell.strip())
    if not ok or not cell.strip():
        raise ValueError("not a number: %r" % cell)
    return v


def read_trajectory(text, species_names):
    """A trajectory export (csvw_sim, io/csvw_sim.ipp:17-91: what
    ``simulation -e`` writes) as the samples the analyses of ``simulation
    -i`` see.

    The header row gives cell-total, time-start, time-col, cell-start,
    cell-end and one 0/1 flag per species; the row of column names gives
    the value columns' species in file order (csvw_sim writes them in the
    -o order, not by species id), after an optional Time (and Cell) column;
    then each sample is cell-end - cell-start rows of values, one row per
    cell.  Numbers are read as DENSE reads them (strtold, then double).
    Returns (header dict, samples [k][num_species][cell_total]) with NaN for
    species and cells the file does not hold."""
    import numpy as np
    lines = [ln.strip() for ln in text.splitlines()]
    body = [ln for ln in lines if ln and not ln.startswith("#")]
    if len(body) < 3 or not body[0].startswith("cell-total"):
        raise ValueError("not a trajectory export: no cell-total header row")
    head = [x for x in body[1].split(",") if x.strip()]
    nsp = len(species_names)
    if len(head) != 5 + nsp:
        raise ValueError("trajectory header has %d fields, expected %d" % (len(head), 5 + nsp))
    nums = [_number(x) for x in head]
    cells, t0, time_col, cs, ce = int(nums[0]), nums[1], int(nums[2]), int(nums[3]), int(nums[4])
    names = [x.strip() for x in body[2].split(",") if x.strip()]
    skip = 0
    while names and names[0] in ("Time", "Cell"):
        names.pop(0)
        skip += 1
    cols = [species_names.index(nm) for nm in names]
    flagged = sorted(i for i in range(nsp) if nums[5 + i] != 0.0)
    if sorted(cols) != flagged:
        raise ValueError("trajectory columns %s do not match the header's species flags" % names)
    m = ce - cs
    rows = []
    for ln in body[3:]:
        cellsv = ln.split(",")
        if cellsv and cellsv[-1].strip() == "":
            cellsv = cellsv[:-1]
        vals = cellsv[skip:]
        if len(vals) != len(cols):
            raise ValueError("trajectory row with %d values, expected %d: %r" % (len(vals), len(cols), ln))
        rows.append([_number(v) for v in vals])
    if m <= 0 or len(rows) % m:
        raise ValueError("trajectory rows (%d) are not whole samples of %d cells" % (len(rows), m))
    k = len(rows) // m
    out = np.full((k, nsp, cells), np.nan)
    R = np.asarray(rows, np.float64).reshape(k, m, len(cols))
    for j, sp in enumerate(cols):
        out[:, sp, cs:ce] = R[:, :, j]
    return {"cell_total": cells, "time_start": t0, "time_col": time_col, "cell_start": cs, "cell_end": ce,
            "species": cols}, out
