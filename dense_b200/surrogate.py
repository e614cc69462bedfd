"""MLP surrogate for the parameter search.

An addition of this project (DENSE's SRES search simulates every candidate,
search/sres.cpp:328-345): a small network maps a candidate's
log-parameters to oscillation features -- log period, log amplitude,
inter-cell synchrony of mh1 and an oscillation indicator -- and
pre-screens candidates, so that only the most promising ones are simulated.
Every candidate it accepts is re-simulated by the FP64 engine, which alone
decides acceptance.

Network: in -> 3 x 256 (GELU) -> out, BF16 weights and activations on the
GEMMs, FP32 accumulation, FP32 master weights with Adam.  Every matrix
product of the forward and backward passes runs in the tcgen05 kernel of
csrc/surrogate/umma_gemm.cuh; torch only allocates the buffers and orders
the launches on one stream.
"""

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_DIR = os.path.join(HERE, "_lib")
SRC = os.path.join(HERE, "csrc", "surrogate")
LIB = os.path.join(LIB_DIR, "libdense_b200_surrogate.so")

EPI_STORE, EPI_BIAS_GELU, EPI_BIAS = 0, 1, 2
HIDDEN = 256
IN_PAD = 64     # input features padded to the GEMM's K granularity
OUT_PAD = 128   # outputs padded to one UMMA M tile for the weight gradient


def build(force=False):
    srcs = [os.path.join(SRC, f) for f in os.listdir(SRC)] + [os.path.join(os.path.dirname(HERE), "include",
                                                                            "dense_b200_surrogate.h")]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs):
        return LIB
    os.makedirs(os.path.join(LIB_DIR, "obj"), exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    base = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3", "-lineinfo",
            "-I", os.path.join(os.path.dirname(HERE), "include")]
    objs = []
    cmds = []
    for unit in ("mlp", "features"):
        obj = os.path.join(LIB_DIR, "obj", unit + ".o")
        objs.append(obj)
        cmds.append(base + ["-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-c",
                            os.path.join(SRC, unit + ".cu"), "-o", obj])
    cmds.append(base + ["-shared", "-o", LIB] + objs + ["-lcudart"])
    for cmd in cmds:
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode:
            raise RuntimeError(r.stderr[-4000:])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(build())
        vp, i, f, i64 = C.c_void_p, C.c_int, C.c_float, C.c_int64
        L.dense_mlp_gemm.argtypes = [vp, i, vp, i, vp, i, i, i, i, i, vp, vp, i, vp, vp]
        L.dense_mlp_gemm_ws.argtypes = [vp, i, vp, i, vp, i, i, i, i, i, vp, vp, i, vp, vp, C.c_size_t, vp]
        L.dense_mlp_transpose_bf16.argtypes = [vp, i, i, i, vp, i, vp]
        L.dense_mlp_cast_bf16.argtypes = [vp, i, i, vp, i, vp]
        L.dense_mlp_gelu_backward.argtypes = [vp, vp, i64, vp, vp, vp]
        L.dense_mlp_mse.argtypes = [vp, i, vp, vp, i, i, f, vp, vp, vp, vp]
        L.dense_mlp_colsum.argtypes = [vp, i, i, vp, vp]
        L.dense_mlp_adam.argtypes = [vp, vp, vp, vp, i64, f, f, f, f, i, vp]
        L.dense_mlp_adam_dev.argtypes = [vp, vp, vp, vp, i64, vp, vp]
        L.dense_mlp_mse_dev.argtypes = [vp, i, vp, vp, i, i, vp, vp, vp, vp, vp]
        L.dense_mlp_gather.argtypes = [vp, i, i, vp, vp, i, vp, i, i, vp, i, vp, vp, vp]
        L.dense_features_synchrony.argtypes = [vp, i64, i64, i, vp, i, vp, vp]
        L.dense_features_encode.argtypes = [vp, i, i, vp, vp, i, C.c_double, vp, i, i, vp]
        L.dense_features_ensemble_accumulate.argtypes = [vp, i, i, i, vp, i, vp]
        L.dense_features_score.argtypes = [vp, i, i, i, vp, vp, C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_double, vp, vp]
        _lib = L
    return _lib


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Kernels:
    """Thin launchers over the C ABI for torch CUDA tensors on one stream.

    The GEMM's split-K workspace (FP32 partials) belongs to this object:
    its launches must stay on one stream."""

    WS_BYTES = 32 << 20

    def __init__(self, device=0):
        import torch
        self.torch = torch
        self.L = lib()
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        self.ws = torch.empty(self.WS_BYTES // 4, dtype=torch.float32, device=self.dev)

    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def gemm(self, A, B, D, epilogue=EPI_STORE, bias=None, H=None):
        """D[M][N] = A[M][K] . B[N][K]^T (BF16 in, FP32 out)."""
        M, K = A.shape
        N = B.shape[0]
        rc = self.L.dense_mlp_gemm_ws(_p(A), A.stride(0), _p(B), B.stride(0), _p(D), D.stride(0), M, N, K, epilogue,
                                      _p(bias), _p(H), H.stride(0) if H is not None else 0, _p(self.err),
                                      _p(self.ws), self.WS_BYTES, self._s())
        if rc:
            raise RuntimeError("dense_mlp_gemm rejected M=%d N=%d K=%d (rc %d)" % (M, N, K, rc))

    def transpose(self, src, dst):
        r, c = src.shape
        assert self.L.dense_mlp_transpose_bf16(_p(src), r, c, src.stride(0), _p(dst), dst.stride(0), self._s()) == 0

    def cast(self, src, dst, transpose=False):
        r, c = src.shape
        assert self.L.dense_mlp_cast_bf16(_p(src), r, c, _p(dst), int(transpose), self._s()) == 0

    def gelu_backward(self, dH, Z, dZ, dZb):
        assert self.L.dense_mlp_gelu_backward(_p(dH), _p(Z), dH.numel(), _p(dZ), _p(dZb), self._s()) == 0

    def mse(self, Y, T, mask, dY, dYb, loss):
        rows, nout = T.shape
        inv = 1.0 / max(1.0, float(mask.sum().item()))
        assert self.L.dense_mlp_mse(_p(Y), Y.stride(0), _p(T), _p(mask), rows, nout, inv, _p(dY), _p(dYb),
                                    _p(loss), self._s()) == 0

    def mse_dev(self, Y, T, mask, inv_count, dY, dYb, loss):
        """mse with the 1 / count scale in a one-element device tensor."""
        rows, nout = T.shape
        assert self.L.dense_mlp_mse_dev(_p(Y), Y.stride(0), _p(T), _p(mask), rows, nout, _p(inv_count), _p(dY),
                                        _p(dYb), _p(loss), self._s()) == 0

    def gather(self, X, T, mask, idx, Xb, Tb, Mb):
        """One batch from a device-resident training set: rows idx of X
        (float [n][n_in]) to BF16 Xb [Bp][in_pad] (zero padded), of T and
        mask to Tb and Mb [Bp][n_out]; rows past len(idx) are zeros."""
        n, n_in = X.shape
        Bp, in_pad = Xb.shape
        assert self.L.dense_mlp_gather(_p(X), n, n_in, _p(T), _p(mask), T.shape[1], _p(idx), idx.shape[0], Bp,
                                       _p(Xb), in_pad, _p(Tb), _p(Mb), self._s()) == 0

    def adam_dev(self, w, g, m, v, hyper):
        """adam with {lr, b1, b2, eps, 1 - b1^t, 1 - b2^t} in device memory."""
        assert self.L.dense_mlp_adam_dev(_p(w), _p(g), _p(m), _p(v), w.numel(), _p(hyper), self._s()) == 0

    def synchrony(self, X, counts, out):
        """Mean pairwise Pearson correlation across cells per set: X a
        float64 CUDA tensor [sets][samples][cells] (cells contiguous; any
        set and sample strides), counts int32 [sets] (samples per set),
        out float64 [sets]."""
        B, _, cells = X.shape
        assert X.stride(2) == 1
        assert self.L.dense_features_synchrony(_p(X), X.stride(0), X.stride(1), cells, _p(counts), B, _p(out),
                                               self._s()) == 0

    def encode(self, P, idx, tmpl, log_spread, Xb):
        """Network inputs of candidates P (float64 [n][params]) into BF16
        Xb [Bp][in_pad]: log(P[:, idx] / tmpl) / log_spread, zero padded."""
        n, ldp = P.shape
        Bp, in_pad = Xb.shape
        assert P.stride(1) == 1
        assert self.L.dense_features_encode(_p(P), P.stride(0), n, _p(idx), _p(tmpl), idx.shape[0], float(log_spread),
                                            _p(Xb), in_pad, Bp, self._s()) == 0

    def ensemble_accumulate(self, Y, n, nout, acc, first):
        assert self.L.dense_features_ensemble_accumulate(_p(Y), Y.stride(0), n, nout, _p(acc), int(first),
                                                         self._s()) == 0

    def score(self, acc, nets, mu, sd, weight, period, tol, amp_min, ramp, out):
        """Ranking score from the ensemble sum acc [n][nout] (see
        csrc/surrogate/features.cu); mu and sd numpy float32 [nout]."""
        n, nout = acc.shape
        mu = np.ascontiguousarray(mu, np.float32)
        sd = np.ascontiguousarray(sd, np.float32)
        assert self.L.dense_features_score(_p(acc), n, nout, nets, mu.ctypes.data_as(C.c_void_p),
                                           sd.ctypes.data_as(C.c_void_p), weight, period, tol, amp_min, ramp, _p(out),
                                           self._s()) == 0

    def colsum(self, dZ, db):
        r, c = dZ.shape
        assert self.L.dense_mlp_colsum(_p(dZ), r, c, _p(db), self._s()) == 0

    def adam(self, w, g, m, v, lr, step, b1=0.9, b2=0.999, eps=1e-8):
        assert self.L.dense_mlp_adam(_p(w), _p(g), _p(m), _p(v), w.numel(), lr, b1, b2, eps, step, self._s()) == 0

    def check(self):
        self.torch.cuda.synchronize(self.dev)
        e = int(self.err.item())
        if e:
            raise RuntimeError("tensor-core GEMM reported error bits %d" % e)


class MLP:
    """in -> 3 x 256 GELU -> out on the tensor-core kernels.

    Weights are kept as FP32 masters [out][in] with Adam moments; every step
    casts them to BF16 (and transposed BF16 copies for the input-gradient
    products).  Inputs are padded to IN_PAD features and outputs to OUT_PAD
    rows (the padding weights stay zero: their gradients are zero).
    """

    def __init__(self, n_in, n_out, seed=0, device=0, lr=1e-3, group=None):
        """`group`: a torch.distributed process group for data-parallel
        training (every rank the same seed, so the same initial weights; the
        gradients of each step are averaged over the ranks)."""
        import torch
        assert n_in <= IN_PAD and n_out <= OUT_PAD
        self.torch = torch
        self.k = Kernels(device)
        self.dev = self.k.dev
        self.n_in, self.n_out, self.lr = n_in, n_out, lr
        rng = np.random.Generator(np.random.PCG64(seed))
        shapes = [(HIDDEN, IN_PAD), (HIDDEN, HIDDEN), (HIDDEN, HIDDEN), (OUT_PAD, HIDDEN)]
        fan_in = [n_in, HIDDEN, HIDDEN, HIDDEN]
        self.W, self.b = [], []
        for i, (o, n) in enumerate(shapes):
            w = np.zeros((o, n), np.float32)
            rows = o if i < 3 else n_out
            cols = n if i > 0 else n_in
            w[:rows, :cols] = rng.normal(0.0, np.sqrt(2.0 / fan_in[i]), size=(rows, cols))
            self.W.append(torch.tensor(w, device=self.dev))
            self.b.append(torch.zeros(o, device=self.dev))
        self.mW = [torch.zeros_like(w) for w in self.W]
        self.vW = [torch.zeros_like(w) for w in self.W]
        self.mb = [torch.zeros_like(b) for b in self.b]
        self.vb = [torch.zeros_like(b) for b in self.b]
        self.steps = 0
        self._bufs = {}
        self.group = group

    def _buf(self, name, shape, dtype=None):
        t = self._bufs.get(name)
        dtype = dtype or self.torch.float32
        if t is None or tuple(t.shape) != tuple(shape) or t.dtype != dtype:
            t = self.torch.empty(shape, dtype=dtype, device=self.dev)
            self._bufs[name] = t
        return t

    def _cast_weights(self):
        bf = self.torch.bfloat16
        self.Wb = [self._buf("Wb%d" % i, w.shape, bf) for i, w in enumerate(self.W)]
        self.WTb = [self._buf("WTb%d" % i, (w.shape[1], w.shape[0]), bf) for i, w in enumerate(self.W)]
        for i, w in enumerate(self.W):
            self.k.cast(w, self.Wb[i])
            if i > 0:
                self.k.cast(w, self.WTb[i], transpose=True)

    def _input(self, X):
        """[B][n_in] float -> padded BF16 [Bp][IN_PAD], Bp a multiple of 128."""
        B = X.shape[0]
        Bp = (B + 127) // 128 * 128
        Xb = self._buf("Xb", (Bp, IN_PAD), self.torch.bfloat16)
        Xb.zero_()
        Xb[:B, :self.n_in] = self.torch.as_tensor(X, device=self.dev, dtype=self.torch.float32).to(self.torch.bfloat16)
        return Xb, Bp

    def forward(self, Xb):
        Bp = Xb.shape[0]
        bf = self.torch.bfloat16
        self.Z = [self._buf("Z%d" % i, (Bp, HIDDEN)) for i in range(3)]
        self.H = [Xb] + [self._buf("H%d" % i, (Bp, HIDDEN), bf) for i in range(1, 4)]
        for i in range(3):
            self.k.gemm(self.H[i], self.Wb[i], self.Z[i], EPI_BIAS_GELU, self.b[i], self.H[i + 1])
        Y = self._buf("Y", (Bp, OUT_PAD))
        self.k.gemm(self.H[3], self.Wb[3], Y, EPI_BIAS, self.b[3])
        return Y

    def predict_device(self, X, batch=65536):
        """Outputs [B][n_out] as a CUDA float32 tensor, for inputs already
        on the GPU (a float tensor [B][n_in]); nothing crosses to the host."""
        torch = self.torch
        self._cast_weights()
        out = []
        for s in range(0, X.shape[0], batch):
            x = X[s:s + batch]
            B = x.shape[0]
            Bp = (B + 127) // 128 * 128
            Xb = self._buf("Xb", (Bp, IN_PAD), torch.bfloat16)
            Xb.zero_()
            Xb[:B, :self.n_in] = x.to(torch.bfloat16)
            Y = self.forward(Xb)
            out.append(Y[:B, :self.n_out].clone())
        self.k.check()
        return torch.cat(out) if out else torch.zeros((0, self.n_out), device=self.dev)

    def predict(self, X, batch=65536):
        """Outputs [B][n_out] (float32, on the host)."""
        self._cast_weights()
        out = []
        for s in range(0, X.shape[0], batch):
            Xb, _ = self._input(X[s:s + batch])
            Y = self.forward(Xb)
            out.append(Y[:min(batch, X.shape[0] - s), :self.n_out].float().cpu().numpy())
        self.k.check()
        return np.concatenate(out) if out else np.zeros((0, self.n_out), np.float32)

    def gradients(self, X, T, mask):
        """Loss and gradients (dW, db lists) of one batch; Bp rows, padding masked."""
        torch = self.torch
        bf = torch.bfloat16
        self._cast_weights()
        Xb, Bp = self._input(X)
        B = X.shape[0]
        Tt = torch.zeros((Bp, self.n_out), device=self.dev)
        Mt = torch.zeros((Bp, self.n_out), device=self.dev)
        Tt[:B] = torch.as_tensor(np.nan_to_num(T), device=self.dev, dtype=torch.float32)
        Mt[:B] = torch.as_tensor(mask, device=self.dev, dtype=torch.float32)
        Y = self.forward(Xb)
        loss = torch.zeros(1, device=self.dev)
        dY = self._buf("dY", (Bp, OUT_PAD))
        dYb = self._buf("dYb", (Bp, OUT_PAD), bf)
        self.k.mse(Y, Tt, Mt, dY, dYb, loss)
        dW, db = self._backward(dY, dYb, Bp)
        self.k.check()
        return float(loss.item()), dW, db

    def _backward(self, dY, dYb, Bp):
        """Weight and bias gradients from the output gradient dY (FP32 and
        BF16 copies) of the last forward pass over Bp rows."""
        bf = self.torch.bfloat16
        dW = [None] * 4
        db = [None] * 4
        dZ, dZb = dY, dYb
        for i in (3, 2, 1, 0):
            rows = self.W[i].shape[0]
            # weight gradient: dW_i = dZ^T H_i  (M = out rows, N = in, K = batch)
            dZT = self._buf("dZT%d" % i, (rows, Bp), bf)
            HT = self._buf("HT%d" % i, (self.W[i].shape[1], Bp), bf)
            self.k.transpose(dZb, dZT)
            self.k.transpose(self.H[i], HT)
            dW[i] = self._buf("dW%d" % i, self.W[i].shape)
            self.k.gemm(dZT, HT, dW[i])
            db[i] = self._buf("db%d" % i, (rows,))
            self.k.colsum(dZ, db[i])
            if i == 0:
                break
            # input gradient: dH_i = dZ W_i, then dZ_{i-1} = dH_i * GELU'(Z_{i-1})
            dH = self._buf("dH%d" % i, (Bp, HIDDEN))
            self.k.gemm(dZb, self.WTb[i], dH)
            ndZ = self._buf("dZ%d" % (i - 1), (Bp, HIDDEN))
            ndZb = self._buf("dZb%d" % (i - 1), (Bp, HIDDEN), bf)
            self.k.gelu_backward(dH, self.Z[i - 1], ndZ, ndZb)
            dZ, dZb = ndZ, ndZb
        return dW, db

    def _train_graphs(self, data, batch, steps):
        """CUDA graphs of training on the device-resident training set
        `data` = (X, T, mask), `steps` steps of `batch` rows per epoch.
        Per epoch the host writes the epoch's row indices ("idx", steps x
        batch) and per-step scalars ("hyper", steps x {lr, b1, b2, eps,
        1 - b1^t, 1 - b2^t, 1 / count}) into static device buffers.  One
        process: one graph replays the whole epoch (per step: batch gather,
        weight casts, forward, loss, backward, Adam).  Data-parallel: per
        step a gradient graph and an update graph, with the gradient
        all-reduce between them.  The graphs hold the addresses of this
        object's work buffers: they serve one fit call only (no other pass
        may resize a buffer meanwhile)."""
        torch = self.torch
        Bp = (batch + 127) // 128 * 128
        bf = torch.bfloat16
        g = {"Bp": Bp}
        g["idx"] = torch.zeros(steps * batch, dtype=torch.int32, device=self.dev)
        g["hyper"] = torch.zeros((steps, 8), device=self.dev)
        g["loss"] = torch.zeros(1, device=self.dev)
        Xd, Td, Md = data

        def grads(j):
            self._cast_weights()
            Xb = self._buf("Xb", (Bp, IN_PAD), bf)
            Tb = self._buf("Tb", (Bp, self.n_out))
            Mb = self._buf("Mb", (Bp, self.n_out))
            self.k.gather(Xd, Td, Md, g["idx"][j * batch:(j + 1) * batch], Xb, Tb, Mb)
            Y = self.forward(Xb)
            dY = self._buf("dY", (Bp, OUT_PAD))
            dYb = self._buf("dYb", (Bp, OUT_PAD), bf)
            self.k.mse_dev(Y, Tb, Mb, g["hyper"][j, 6:7], dY, dYb, g["loss"])
            g["dW"], g["db"] = self._backward(dY, dYb, Bp)

        def update(j):
            hyper = g["hyper"][j]
            for i in range(4):
                self.k.adam_dev(self.W[i], g["dW"][i], self.mW[i], self.vW[i], hyper)
                self.k.adam_dev(self.b[i], g["db"][i], self.mb[i], self.vb[i], hyper)

        side = torch.cuda.Stream(self.dev)
        side.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(side):
            grads(0)  # allocates every buffer before capture; changes no weight
        torch.cuda.current_stream(self.dev).wait_stream(side)
        torch.cuda.synchronize(self.dev)
        if self.group is None:
            g["epoch"] = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g["epoch"]):
                for j in range(steps):
                    grads(j)
                    update(j)
        else:
            g["grads"], g["update"] = [], []
            for j in range(steps):
                gg, gu = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
                with torch.cuda.graph(gg):
                    grads(j)
                with torch.cuda.graph(gu):
                    update(j)
                g["grads"].append(gg)
                g["update"].append(gu)
        return g

    def _fit_epochs(self, X, T, mask, n, epochs, batch, rng, cosine, data=None, b1=0.9, b2=0.999, eps=1e-8):
        """Generator behind the captured fit: each next() enqueues one epoch
        on the current stream and returns a function that reads that
        epoch's mean loss (call it before the next epoch is enqueued).
        `data`: the training set already on the device (X, T, mask)."""
        torch = self.torch
        steps = n // batch
        if steps == 0:
            for _ in range(epochs):
                yield lambda: 0.0
            return
        if data is None:
            data = device_training_set(X, T, mask, self.dev)
        g = self._train_graphs(data, batch, steps)
        lr0 = self.lr
        total = epochs * steps
        for ep in range(epochs):
            rows = rng.permutation(X.shape[0])[:n][:steps * batch]
            counts = mask[rows].reshape(steps, batch, -1).sum(axis=(1, 2), dtype=np.float64)
            hyp = np.zeros((steps, 8), np.float64)
            for j in range(steps):
                lr = lr0
                if cosine:
                    t = (ep * steps + j) / max(1, total - 1)
                    lr = lr0 * (0.01 + 0.99 * 0.5 * (1.0 + np.cos(np.pi * t)))
                step = self.steps + j + 1
                hyp[j] = (lr, b1, b2, eps, 1.0 - b1 ** step, 1.0 - b2 ** step, 1.0 / max(1.0, counts[j]), 0.0)
            g["idx"].copy_(torch.as_tensor(rows.astype(np.int32)))
            g["hyper"].copy_(torch.as_tensor(hyp.astype(np.float32)))
            g["loss"].zero_()
            if self.group is None:
                g["epoch"].replay()
            else:
                from .distributed import average_
                for j in range(steps):
                    g["grads"][j].replay()
                    average_(g["dW"] + g["db"], self.group)
                    g["update"][j].replay()
            self.steps += steps
            yield lambda: float(g["loss"].item()) / steps
        del g

    def _fit_captured(self, X, T, mask, n, epochs, batch, rng, log, cosine):
        hist = []
        for ep, loss in enumerate(self._fit_epochs(X, T, mask, n, epochs, batch, rng, cosine)):
            hist.append(loss())
            self.k.check()
            if log:
                log("epoch %d loss %.5f" % (ep, hist[-1]))
        return hist

    def step(self, X, T, mask):
        loss, dW, db = self.gradients(X, T, mask)
        if self.group is not None:
            from .distributed import average_
            average_(dW + db, self.group)
        self.steps += 1
        for i in range(4):
            self.k.adam(self.W[i], dW[i], self.mW[i], self.vW[i], self.lr, self.steps)
            self.k.adam(self.b[i], db[i], self.mb[i], self.vb[i], self.lr, self.steps)
        return loss

    def fit(self, X, T, mask, epochs=20, batch=4096, seed=0, log=None, cosine=True, captured=True):
        """Minibatch Adam; with `cosine` the learning rate follows a cosine
        from lr down to lr/100 over the run.  With `captured` (the default)
        the training set is copied to the GPU once and every step replays
        two CUDA graphs (gradient, update); otherwise each step is launched
        from the host (`step`), with the same batches and schedule."""
        rng = np.random.Generator(np.random.PCG64(seed))
        n = X.shape[0]
        if self.group is not None:
            # every rank takes the same number of steps: the smallest shard's
            import torch.distributed as dist
            t = self.torch.tensor([n], device=self.dev)
            dist.all_reduce(t, op=dist.ReduceOp.MIN, group=self.group)
            n = int(t.item())
        if captured:
            return self._fit_captured(X, T, mask, n, epochs, batch, rng, log, cosine)
        hist = []
        lr0 = self.lr
        per_epoch = max(1, n // batch)
        total = epochs * per_epoch
        for ep in range(epochs):
            order = rng.permutation(X.shape[0])[:n]
            tot = 0.0
            for j, s in enumerate(range(0, n - batch + 1, batch)):
                if cosine:
                    t = (ep * per_epoch + j) / max(1, total - 1)
                    self.lr = lr0 * (0.01 + 0.99 * 0.5 * (1.0 + np.cos(np.pi * t)))
                idx = order[s:s + batch]
                tot += self.step(X[idx], T[idx], mask[idx])
            hist.append(tot / max(1, n // batch))
            if log:
                log("epoch %d loss %.5f" % (ep, hist[-1]))
        self.lr = lr0
        return hist

    def state(self):
        return {"W": [w.cpu().numpy() for w in self.W], "b": [b.cpu().numpy() for b in self.b]}


def device_training_set(X, T, mask, dev):
    """The training set on the device as float32 tensors (NaN targets 0)."""
    import torch
    return (torch.as_tensor(np.ascontiguousarray(X, dtype=np.float32), device=dev),
            torch.as_tensor(np.ascontiguousarray(np.nan_to_num(T), dtype=np.float32), device=dev),
            torch.as_tensor(np.ascontiguousarray(mask, dtype=np.float32), device=dev))


def fit_concurrently(nets, X, T, mask, seeds, epochs=20, batch=4096, log=None, cosine=True):
    """MLP.fit of several networks of one process at once, each on its own
    CUDA stream (a network's epoch is one graph replay; the GEMMs of one
    4096-row batch fill only a few dozen SMs, so the networks share the
    GPU).  Network k takes the batches of seed seeds[k]: its weights are
    those of nets[k].fit(..., seed=seeds[k]).  Returns the loss histories."""
    import torch
    assert all(net.group is None for net in nets)
    dev = nets[0].dev
    data = device_training_set(X, T, mask, dev)
    n = X.shape[0]
    streams = [torch.cuda.Stream(dev) for _ in nets]
    for st in streams:
        st.wait_stream(torch.cuda.current_stream(dev))
    gens = [net._fit_epochs(X, T, mask, n, epochs, batch, np.random.Generator(np.random.PCG64(sd)), cosine,
                            data=data) for net, sd in zip(nets, seeds)]
    hists = [[] for _ in nets]
    for ep in range(epochs):
        readers = []
        for gen, st in zip(gens, streams):
            with torch.cuda.stream(st):
                readers.append(next(gen))
        for k, (read, st) in enumerate(zip(readers, streams)):
            with torch.cuda.stream(st):
                hists[k].append(read())
        for net in nets:
            net.k.check()
        if log:
            log("epoch %d loss %s" % (ep, " ".join("%.5f" % h[-1] for h in hists)))
    for gen in gens:
        gen.close()
    torch.cuda.current_stream(dev).wait_stream(streams[0])
    for st in streams[1:]:
        torch.cuda.current_stream(dev).wait_stream(st)
    return hists


def bench_gemm(rows=131072, reps=20, device=0):
    """Times the tensor-core GEMM on the MLP's layer shapes (BF16 inputs,
    FP32 outputs): rows x 256 x 64 (first layer), rows x 256 x 256 (hidden
    layers), rows x 128 x 256 (output layer), plain and with the bias+GELU
    epilogue; one dict per shape and epilogue, CUDA-event timed."""
    import torch
    k = Kernels(device)
    dev = "cuda:%d" % device
    out = []
    for (n, kk) in ((256, 64), (256, 256), (128, 256)):
        A = torch.randn(rows, kk, device=dev).to(torch.bfloat16)
        B = torch.randn(n, kk, device=dev).to(torch.bfloat16)
        D = torch.empty(rows, n, device=dev, dtype=torch.float32)
        H = torch.empty(rows, n, device=dev, dtype=torch.bfloat16)
        bias = torch.randn(n, device=dev)
        for epi, name in ((EPI_STORE, "store"), (EPI_BIAS_GELU, "bias_gelu")):
            k.gemm(A, B, D, epi, bias, H)
            torch.cuda.synchronize(device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s = torch.cuda.current_stream(device)
            e0.record(s)
            for _ in range(reps):
                k.gemm(A, B, D, epi, bias, H)
            e1.record(s)
            torch.cuda.synchronize(device)
            ms = e0.elapsed_time(e1) / reps
            nbytes = rows * kk * 2 + n * kk * 2 + rows * n * 4 + (rows * n * 2 if epi == EPI_BIAS_GELU else 0)
            out.append({"rows": rows, "n": n, "k": kk, "epilogue": name, "us": ms * 1e3,
                        "tflops": 2.0 * rows * n * kk / ms / 1e9, "gbs": nbytes / ms / 1e6})
    k.check()
    return out


def bench_fit(rows=200000, epochs=3, batch=4096, n_in=44, n_out=5, device=0):
    """Wall time per training step of MLP.fit on seeded random data, the
    captured form (one CUDA graph per epoch) and the launched form; each
    after a one-epoch warm-up on a slice, graph capture included."""
    import time
    import torch
    rng = np.random.Generator(np.random.PCG64(0))
    X = rng.uniform(-1, 1, size=(rows, n_in)).astype(np.float32)
    T = rng.normal(size=(rows, n_out)).astype(np.float32)
    M = np.ones((rows, n_out), np.float32)
    out = []
    for captured in (True, False):
        net = MLP(n_in, n_out, seed=0, device=device)
        net.fit(X[:8 * batch], T[:8 * batch], M[:8 * batch], epochs=1, batch=batch, captured=captured)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        net.fit(X, T, M, epochs=epochs, batch=batch, captured=captured)
        torch.cuda.synchronize(device)
        steps = epochs * (rows // batch)
        out.append({"captured": captured, "rows": rows, "batch": batch, "epochs": epochs, "steps": steps,
                    "ms_per_step": 1e3 * (time.perf_counter() - t0) / steps})
    return out


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="time the surrogate's tensor-core GEMM, or its training steps")
    ap.add_argument("--rows", type=int, default=131072)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--fit", action="store_true", help="time MLP.fit steps instead (--rows training rows)")
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=4096)
    a = ap.parse_args()
    for r in (bench_fit(a.rows, a.epochs, a.batch) if a.fit else bench_gemm(a.rows, a.reps)):
        print(json.dumps(r))
