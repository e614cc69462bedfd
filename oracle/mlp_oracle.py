"""ORACLE -- test infrastructure only.

The surrogate MLP in plain numpy float64: forward pass, masked mean
squared error and its gradients by the chain rule, for checking the
tensor-core training kernels (dense_b200/surrogate.py) on the same weights
and inputs.  GELU is the exact form x * Phi(x).
"""

import math

import numpy as np

_erf = np.vectorize(math.erf)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def loss_and_grads(W, b, X, T, mask):
    """W[i]: [out][in], b[i]: [out]; X [B][in]; T, mask [B][n_out] (n_out
    <= rows of the last layer).  Returns loss, dW, db."""
    W = [np.asarray(w, np.float64) for w in W]
    b = [np.asarray(v, np.float64) for v in b]
    H = [np.asarray(X, np.float64)]
    Z = []
    for i in range(3):
        Z.append(H[-1] @ W[i].T + b[i])
        H.append(gelu(Z[-1]))
    Y = H[-1] @ W[3].T + b[3]
    n_out = T.shape[1]
    count = max(1.0, float(mask.sum()))
    d = (Y[:, :n_out] - np.nan_to_num(T)) * mask
    loss = float((d * (Y[:, :n_out] - np.nan_to_num(T))).sum() / count)
    dZ = np.zeros_like(Y)
    dZ[:, :n_out] = 2.0 * d / count
    dW, db = [None] * 4, [None] * 4
    for i in (3, 2, 1, 0):
        dW[i] = dZ.T @ H[i]
        db[i] = dZ.sum(axis=0)
        if i:
            dZ = (dZ @ W[i]) * gelu_grad(Z[i - 1])
    return loss, dW, db
