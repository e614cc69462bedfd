"""Uneven mixed batches: sets of several models in one captured CUDA graph.

Each model is its own engine library (the model is compiled in, as in
DENSE), so a mixed batch holds one engine per model.  ``MixedBatch.run``
replays one CUDA graph that forks every engine's launches onto a stream of
its own and joins them back, so the models' kernels share the GPU; each
engine in turn forks its register-kernel and memory-kernel groups.  A step
of ``num_chunks`` analysis intervals advances every unfinished set.
"""

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
        self._streams = None

    def _capture(self, num_chunks):
        import torch
        if self._streams is None:
            self._streams = [torch.cuda.Stream(device=self.device) for _ in self.batches]
            self._main = torch.cuda.Stream(device=self.device)
        # a launch of zero chunks outside capture sets every kernel attribute
        for b in self.batches.values():
            b.run(0, stream=self._main.cuda_stream)
        self._main.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self._main, capture_error_mode="thread_local"):
            for st, b in zip(self._streams, self.batches.values()):
                st.wait_stream(self._main)
                b.run(num_chunks, stream=st.cuda_stream)
            for st in self._streams:
                self._main.wait_stream(st)
        return g

    def run(self, num_chunks, stream=None):
        """Replay the graph that advances every set by `num_chunks` chunks
        (captured on first use) on `stream` (a torch stream)."""
        import torch
        g = self._graphs.get(num_chunks)
        if g is None:
            g = self._graphs[num_chunks] = self._capture(num_chunks)
        if stream is None:
            g.replay()
        else:
            with torch.cuda.stream(stream):
                g.replay()

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
        self._graphs.clear()
        for b in self.batches.values():
            b.close()
