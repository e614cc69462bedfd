"""Uneven mixed batches: sets of several models in one captured CUDA graph.

Each model is its own engine library (the model is compiled in, as in
DENSE), so a mixed batch holds one engine per model.  ``MixedBatch.run``
replays one CUDA graph (dense_graph_capture) that forks every engine onto a
branch of its own; each engine in turn forks its kernel groups onto streams
prioritised by their longest sets, so the models' kernels share the GPU and
the longest sets start first.  A step of ``num_chunks`` analysis intervals
advances every unfinished set.
"""

import ctypes as C

import numpy as np

from . import engine as E


class MixedBatch:
    def __init__(self, groups, step_size, analysis_interval, analyses=None, precision=E.FP64, device=0):
        """groups: {model: [ParameterSet]}; analyses: {model: [Analysis]}."""
        analyses = analyses or {}
        self.device = device
        self.batches = {m: E.Batch(m, sets, step_size, analysis_interval, analyses.get(m, ()), precision, device)
                        for m, sets in groups.items() if sets}
        self._graphs = {}

    def _capture(self, num_chunks):
        bs = list(self.batches.values())
        # a launch of zero chunks outside capture sets every kernel attribute
        for b in bs:
            b.run(0)
        for b in bs:
            b.sync()
        fns = (C.c_void_p * len(bs))(*[C.cast(b.L.lib.dense_engine_run, C.c_void_p).value for b in bs])
        engs = (C.c_void_p * len(bs))(*[b.h.value for b in bs])
        g = C.c_void_p()
        L = bs[0].L
        L._check(L.lib.dense_graph_capture(len(bs), fns, engs, int(num_chunks), self.device, C.byref(g)))
        return g

    def run(self, num_chunks, stream=None):
        """Replay the graph that advances every set by `num_chunks` chunks
        (captured on first use) on `stream` (a torch stream, or None for the
        default stream)."""
        g = self._graphs.get(num_chunks)
        if g is None:
            g = self._graphs[num_chunks] = self._capture(num_chunks)
        L = next(iter(self.batches.values())).L
        L._check(L.lib.dense_graph_launch(g, None if stream is None else C.c_void_p(stream.cuda_stream)))

    def sync(self):
        """Wait for every launch on the device."""
        import torch
        torch.cuda.synchronize(self.device)

    def reset(self):
        for b in self.batches.values():
            b.reset()
        for b in self.batches.values():
            b.sync()

    def info(self):
        out = {"total_cell_steps": 0, "device_bytes": 0}
        for b in self.batches.values():
            i = b.info()
            out["total_cell_steps"] += i["total_cell_steps"]
            out["device_bytes"] += i["device_bytes"]
        return out

    def done_cell_steps(self, steps_per_chunk):
        """Cell-steps run so far, from every set's chunk counter."""
        total = 0
        for b in self.batches.values():
            chunks, _ = b.progress()
            cells = np.array([s.num_cells for s in b.sets], np.int64)
            total += int((chunks.astype(np.int64) * steps_per_chunk * cells).sum())
        return total

    def close(self):
        if self.batches:
            L = next(iter(self.batches.values())).L
            for g in self._graphs.values():
                L.lib.dense_graph_destroy(g)
        self._graphs.clear()
        for b in self.batches.values():
            b.close()
