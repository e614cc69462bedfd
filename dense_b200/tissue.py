"""Tissue graphs as CSR neighbour lists.

DENSE keeps each cell's out-neighbours in a std::set (NGraph tGraph,
ngraph/ngraph.hpp:80-135), so neighbour ids ascend; the engine takes the same
order, since the neighbour average sums in it (determ.hpp:81-89).
"""

import numpy as np


def default_graph(cell_total, tissue_width):
    """DENSE's default tissue (create_default_graph, Sim_Initializer.hpp:103-136).

    A hexagonal stencil with periodic wrap and directed out-edges: cells on
    the first column get top, top-left, top-right and bottom-left, cells on
    the last column top, top-right, bottom-right and bottom, the rest
    top-right, bottom-right, bottom, top-left and bottom-left; duplicates and
    self-loops collapse as in a std::set.  Returns (offsets, ids) int32.
    """
    n, w = int(cell_total), int(tissue_width)
    if n <= 0 or w <= 0:
        raise ValueError("cell_total and tissue_width must be positive")
    out = []
    for i in range(n):
        former = i % w == 0
        latter = (i + 1) % w == 0
        even = i % 2 == 0
        la = w - 1 if (former or not even) else -1
        ra = w + 1 if not (latter or even) else 1
        top = (i - w + n) % n
        bottom = (i + w) % n
        bottom_right = (i + ra) % n
        top_left = (i + la) % n
        top_right = (i - w + ra + n) % n
        bottom_left = (i - w + la + n) % n
        if former:
            nb = [top, top_left, top_right, bottom_left]
        elif latter:
            nb = [top, top_right, bottom_right, bottom]
        else:
            nb = [top_right, bottom_right, bottom, top_left, bottom_left]
        out.append(sorted(set(abs(x) for x in nb)))
    off = np.zeros(n + 1, np.int32)
    for i, nb in enumerate(out):
        off[i + 1] = off[i] + len(nb)
    ids = np.array([x for nb in out for x in nb], np.int32)
    return off, ids


def from_edges(num_cells, edges):
    """CSR from directed (src, dst) pairs; duplicates collapse, ids ascend
    (NGraph's insert_edge keeps a set per vertex)."""
    nb = [set() for _ in range(num_cells)]
    for a, b in edges:
        nb[int(a)].add(int(b))
    off = np.zeros(num_cells + 1, np.int32)
    for i in range(num_cells):
        off[i + 1] = off[i] + len(nb[i])
    ids = np.array([x for s in nb for x in sorted(s)], np.int32)
    return off, ids
