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
