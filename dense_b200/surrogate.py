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
    srcs = [os.path.join(SRC, f) for f in os.listdir(SRC)]
    if not force and os.path.exists(LIB) and all(os.path.getmtime(s) <= os.path.getmtime(LIB) for s in srcs):
        return LIB
    os.makedirs(os.path.join(LIB_DIR, "obj"), exist_ok=True)
    obj = os.path.join(LIB_DIR, "obj", "mlp.o")
    nvcc = os.environ.get("NVCC", "nvcc")
    base = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++17", "-O3", "-lineinfo"]
    for cmd in (base + ["-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "-c",
                        os.path.join(SRC, "mlp.cu"), "-o", obj],
                base + ["-shared", "-o", LIB, obj, "-lcudart"]):
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
        L.dense_mlp_transpose_bf16.argtypes = [vp, i, i, i, vp, i, vp]
        L.dense_mlp_cast_bf16.argtypes = [vp, i, i, vp, i, vp]
        L.dense_mlp_gelu_backward.argtypes = [vp, vp, i64, vp, vp, vp]
        L.dense_mlp_mse.argtypes = [vp, i, vp, vp, i, i, f, vp, vp, vp, vp]
        L.dense_mlp_colsum.argtypes = [vp, i, i, vp, vp]
        L.dense_mlp_adam.argtypes = [vp, vp, vp, vp, i64, f, f, f, f, i, vp]
        _lib = L
    return _lib


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class Kernels:
    """Thin launchers over the C ABI for torch CUDA tensors on one stream."""

    def __init__(self, device=0):
        import torch
        self.torch = torch
        self.L = lib()
        self.dev = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=self.dev)

    def _s(self):
        return C.c_void_p(self.torch.cuda.current_stream(self.dev).cuda_stream)

    def gemm(self, A, B, D, epilogue=EPI_STORE, bias=None, H=None):
        """D[M][N] = A[M][K] . B[N][K]^T (BF16 in, FP32 out)."""
        M, K = A.shape
        N = B.shape[0]
        rc = self.L.dense_mlp_gemm(_p(A), A.stride(0), _p(B), B.stride(0), _p(D), D.stride(0), M, N, K, epilogue,
                                   _p(bias), _p(H), H.stride(0) if H is not None else 0, _p(self.err), self._s())
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
