"""DENSE's analysis CSV text, byte for byte.

DENSE writes analysis results through csvw (io/csvw.cpp): values go to a
std::ostream with default formatting, i.e. printf's %g with 6 significant
digits, and csvw::add_data appends a comma.  The layouts are those of
Analysis<>::show (measurement/base.hpp:40-51), BasicAnalysis::show
(basic.ipp:61-75) and OscillationAnalysis::show (oscillation.ipp:30-77).
"""

import math


def fmt(x):
    """A double as `std::ostream << x` prints it (glibc: negative NaN is
    "-nan"; NaNs made by arithmetic on x86-64 carry the sign bit)."""
    x = float(x)
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    if math.isinf(x):
        return "-inf" if x < 0 else "inf"
    return "%g" % x


def _header(cell_start, cell_end, time_start, time):
    s = "# Showing cells %d-%d" % (cell_start, cell_end)
    if time_start != 0.0:
        s += " between " + fmt(time_start) + " min and "
    else:
        s += " until "
    return s + fmt(time) + " min\n"


def basic_csv(species_names, species_ids, result, cell_start, cell_end, time_start=0.0):
    """BasicAnalysis::show.  `result` holds mins/sums/maxs indexed by
    observation order, samples and time.  DENSE indexes its vectors by
    species id here (basic.ipp:69-72); an id past the observed count reads
    out of bounds in DENSE and is written as nan."""
    out = _header(cell_start, cell_end, time_start, result["time"])
    out += "Species,Minimum Concentration,Mean Concentration,Maximum Concentration\n"
    n = len(species_ids)
    denom = result["samples"] * (cell_end - cell_start)
    for sp in species_ids:
        if sp < n:
            mn, sm, mx = result["mins"][sp], result["sums"][sp], result["maxs"][sp]
            mean = sm / denom if denom != 0 else (math.nan if sm == 0 else math.copysign(math.inf, sm))
        else:
            mn = sm = mx = mean = float("nan")
        out += "%s,%s,%s,%s\n" % (species_names[sp], fmt(mn), fmt(mean), fmt(mx))
    return out


def oscillation_csv(species_names, species_ids, result, cell_start, cell_end, time_start=0.0):
    """OscillationAnalysis::show: per cell, avg peak / avg amp / avg per
    rows.  `result` arrays are [observed species][cell - cell_start]."""
    out = _header(cell_start, cell_end, time_start, result["time"])
    for c in range(cell_end - cell_start):
        out += "\n# Showing cell %d\nSpecies" % (c + cell_start)
        for sp in species_ids:
            out += "," + species_names[sp]
        for label, key in (("avg peak", "avg_peak"), ("avg amp", "amps"), ("avg per", "pers")):
            out += "\n%s," % label
            for s in range(len(species_ids)):
                out += fmt(result[key][s][c]) + ","
    return out
