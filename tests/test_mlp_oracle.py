"""The float64 MLP oracle that the tensor-core training kernels are checked
against, pinned by central finite differences of its own loss: every
gradient it returns matches the numerical derivative."""

import numpy as np

from oracle.mlp_oracle import gelu, gelu_grad, loss_and_grads


def _net(rng, n_in=6, hidden=5, n_out=3, rows=None):
    dims = [n_in, hidden, hidden, hidden, rows or n_out]
    W = [rng.normal(0, 0.6, size=(dims[i + 1], dims[i])) for i in range(4)]
    b = [rng.normal(0, 0.2, size=dims[i + 1]) for i in range(4)]
    return W, b


def test_gelu_derivative():
    z = np.linspace(-4, 4, 81)
    h = 1e-6
    num = (gelu(z + h) - gelu(z - h)) / (2 * h)
    assert np.allclose(gelu_grad(z), num, rtol=1e-7, atol=1e-9)
    assert abs(gelu(np.array([0.0]))[0]) == 0.0 and abs(gelu(np.array([10.0]))[0] - 10.0) < 1e-12


def test_gradients_match_finite_differences():
    rng = np.random.Generator(np.random.PCG64(8))
    # the last layer has more rows than outputs (padding the kernels use)
    W, b = _net(rng, rows=4)
    X = rng.normal(size=(7, 6))
    T = rng.normal(size=(7, 3))
    T[2, 1] = np.nan                      # a missing target ...
    mask = (rng.random((7, 3)) > 0.2).astype(np.float64)
    mask[2, 1] = 0.0                      # ... is masked out
    loss, dW, db = loss_and_grads(W, b, X, T, mask)
    h = 1e-6

    def loss_at(W2, b2):
        return loss_and_grads(W2, b2, X, T, mask)[0]

    for i in range(4):
        for idx in np.ndindex(W[i].shape):
            Wp = [w.copy() for w in W]
            Wm = [w.copy() for w in W]
            Wp[i][idx] += h
            Wm[i][idx] -= h
            num = (loss_at(Wp, b) - loss_at(Wm, b)) / (2 * h)
            assert abs(dW[i][idx] - num) <= 1e-6 * (1.0 + abs(num)), (i, idx, dW[i][idx], num)
        for j in range(b[i].size):
            bp = [v.copy() for v in b]
            bm = [v.copy() for v in b]
            bp[i][j] += h
            bm[i][j] -= h
            num = (loss_at(W, bp) - loss_at(W, bm)) / (2 * h)
            assert abs(db[i][j] - num) <= 1e-6 * (1.0 + abs(num)), (i, j)
    # padding rows of the last layer get no gradient
    assert not dW[3][3].any() and db[3][3] == 0.0
    assert np.isfinite(loss) and loss > 0
