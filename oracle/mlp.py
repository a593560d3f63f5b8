"""Test infrastructure only: numpy restatement of the rank predictor's network.

The learned rank predictor has no counterpart in the reference (which always computes
every eigenpair with LAPACK ?hegv, src/eigensolver.cpp:188-216), so its oracle is this
plain FP64 statement of the network the GPU kernels implement: features standardised with
the model's mean and standard deviation, 64 -> 128 -> 128 -> 1 with ReLU, loss
(1/n) sum_i (out_i - y_i)^2, and the gradient of that loss by backpropagation. It is
pinned by finite differences (tests/test_oracle.py) and checks the GPU's forward pass and
gradient (tests/test_gpu_rank.py). Model layout (floats): mean [64], sd [64], W1 [64][128],
b1 [128], W2 [128][128], b2 [128], W3 [128], b3.
"""
from __future__ import annotations

import numpy as np

F, H = 64, 128
OFF = {"mu": 0, "sd": F, "W1": 2 * F}
OFF["b1"] = OFF["W1"] + F * H
OFF["W2"] = OFF["b1"] + H
OFF["b2"] = OFF["W2"] + H * H
OFF["W3"] = OFF["b2"] + H
OFF["b3"] = OFF["W3"] + H
N_PARAMS = OFF["b3"] + 1


def unpack(model):
    m = np.asarray(model, dtype=np.float64)
    return {"mu": m[OFF["mu"]:OFF["mu"] + F], "sd": m[OFF["sd"]:OFF["sd"] + F],
            "W1": m[OFF["W1"]:OFF["b1"]].reshape(F, H), "b1": m[OFF["b1"]:OFF["W2"]],
            "W2": m[OFF["W2"]:OFF["b2"]].reshape(H, H), "b2": m[OFF["b2"]:OFF["W3"]],
            "W3": m[OFF["W3"]:OFF["b3"]], "b3": m[OFF["b3"]]}


def forward(model, X):
    """(out [n], cache) for features X [n, 64]."""
    p = unpack(model)
    xn = (np.asarray(X, dtype=np.float64) - p["mu"]) / p["sd"]
    z1 = xn @ p["W1"] + p["b1"]
    h1 = np.maximum(z1, 0.0)
    z2 = h1 @ p["W2"] + p["b2"]
    h2 = np.maximum(z2, 0.0)
    out = h2 @ p["W3"] + p["b3"]
    return out, (xn, h1, h2)


def loss_and_gradient(model, X, y):
    """Loss (1/n) sum (out - y)^2 and its gradient with respect to every model float
    (zero for the fixed mean and sd)."""
    p = unpack(model)
    out, (xn, h1, h2) = forward(model, X)
    n = out.shape[0]
    diff = out - np.asarray(y, dtype=np.float64)
    loss = float(np.sum(diff * diff) / n)
    g = 2.0 * diff / n                      # dL/dout
    grad = np.zeros(N_PARAMS)
    grad[OFF["W3"]:OFF["b3"]] = h2.T @ g
    grad[OFF["b3"]] = g.sum()
    dz2 = np.outer(g, p["W3"]) * (h2 > 0)
    grad[OFF["W2"]:OFF["b2"]] = (h1.T @ dz2).reshape(-1)
    grad[OFF["b2"]:OFF["W3"]] = dz2.sum(0)
    dz1 = (dz2 @ p["W2"].T) * (h1 > 0)
    grad[OFF["W1"]:OFF["b1"]] = (xn.T @ dz1).reshape(-1)
    grad[OFF["b1"]:OFF["W2"]] = dz1.sum(0)
    return loss, grad


def features(C, threshold=0.0):
    """The 64 features of a whitened matrix C (n x n Hermitian), as the GPU forms them
    from its lower triangle: the 32 largest |C_ii|, the 16 largest row norms, then
    log(n)/log(4096), trace, threshold, fraction of C_ii above the threshold, sum |C_ii|,
    sum C_ii^2 / |C|_F^2, max row norm^2 / |C|_F^2, sum row norm^4 / |C|_F^4,
    trace / (|C|_F sqrt(n)), fraction of rows with norm^2 above |C|_F^2 / n, sum of C_ii
    above the threshold, C_ii at the ranks n/8, n/4, n/2, 3n/4 (descending), and the share
    of |C|_F^2 in the 16 largest rows; quantities with the unit of C divided by |C|_F."""
    C = np.asarray(C, dtype=np.complex128)
    n = C.shape[0]
    f = np.zeros(F)
    dg = C.diagonal().real
    r2 = (np.abs(C) ** 2).sum(1)
    fro2 = r2.sum()
    if not fro2 > 0:
        return f
    fro = np.sqrt(fro2)
    a = np.sort(np.abs(dg))[::-1][:32]
    f[:a.size] = a / fro
    r = np.sqrt(np.sort(r2)[::-1][:16])
    f[32:32 + r.size] = r / fro
    f[48] = np.log(n) / np.log(4096.0)
    f[49] = dg.sum() / fro
    f[50] = threshold / fro
    f[51] = np.count_nonzero(dg > threshold) / n
    f[52] = np.abs(dg).sum() / fro
    f[53] = (dg ** 2).sum() / fro2
    f[54] = r2.max() / fro2
    f[55] = (r2 ** 2).sum() / fro2 ** 2
    f[56] = dg.sum() / (fro * np.sqrt(n))
    f[57] = np.count_nonzero(r2 > fro2 / n) / n
    f[58] = dg[dg > threshold].sum() / fro
    sd = np.sort(dg)[::-1]
    for k, q in enumerate((n // 8, n // 4, n // 2, (3 * n) // 4)):
        f[59 + k] = sd[q] / fro
    f[63] = (r[:16] ** 2).sum() / fro2
    return f
