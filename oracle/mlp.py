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


def probe_sign(i, p):
    """Rademacher entry (row i, probe p) of the trace-estimate probes, the integer hash the
    GPU uses (32-bit arithmetic)."""
    m = 0xFFFFFFFF
    h = ((i * 0x9E3779B1) & m) ^ ((p * 0x85EBCA77 + 0x165667B1) & m)
    h ^= h >> 15
    h = (h * 0x2C1B3C6D) & m
    h ^= h >> 12
    return 1.0 if (h & 1) else -1.0


def features(C, threshold=0.0, probes=8):
    """The 64 features of a whitened matrix C (n x n Hermitian), as the GPU forms them from
    its lower triangle, with f = |C|_F: the 32 largest |C_ii| / f; log(n)/log(4096); trace /
    f; threshold / f; fraction of C_ii above the threshold; sum |C_ii| / f; sum C_ii^2 /
    f^2; largest squared row norm / f^2; sum of row norms^4 / f^4; fraction of rows with
    squared norm above f^2 / n; sum of C_ii above the threshold / f; C_ii at the ranks n/8,
    n/4, n/2, 3n/4 (descending) / f; then the spectral moments t_k = mean over the probes z
    of z^H C^k z (k = 1..6) and their combinations (t3 / f^3, t4 / f^4, t5 / f^5, t6 / f^6,
    effective ranks f^4 / t4 and (f^6 / t6)^(1/2) over n, t4^2 / (t6 f^2), t3^2 / (t4 f^2),
    t5 / (t4 f), the effective ranks' logarithms / log(n), t1 t3 / f^4, t3 / (f t4^(1/2)),
    t5 / (t4 t6)^(1/2), t2 / f^2, t1 / f, and their ratio); last, the 16 largest rows'
    share of f^2."""
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
    ln = np.log(n)
    f[32] = ln / np.log(4096.0)
    f[33] = dg.sum() / fro
    f[34] = threshold / fro
    f[35] = np.count_nonzero(dg > threshold) / n
    f[36] = np.abs(dg).sum() / fro
    f[37] = (dg ** 2).sum() / fro2
    f[38] = r2.max() / fro2
    f[39] = (r2 ** 2).sum() / fro2 ** 2
    f[40] = np.count_nonzero(r2 > fro2 / n) / n
    f[41] = dg[dg > threshold].sum() / fro
    sd = np.sort(dg)[::-1]
    for k, q in enumerate((n // 8, n // 4, n // 2, (3 * n) // 4)):
        f[42 + k] = sd[q] / fro
    if probes:
        Z = np.array([[probe_sign(i, p) for p in range(probes)] for i in range(n)])
        Y1 = C @ Z
        Y2 = C @ Y1
        Y3 = C @ Y2
        t1 = np.sum(Z * Y1.real) / probes
        t2 = np.sum(np.abs(Y1) ** 2) / probes
        t3 = np.sum((np.conj(Y1) * Y2).real) / probes
        t4 = np.sum(np.abs(Y2) ** 2) / probes
        t5 = np.sum((np.conj(Y2) * Y3).real) / probes
        t6 = np.sum(np.abs(Y3) ** 2) / probes
        er4, er6 = fro2 ** 2 / t4, np.sqrt(fro2 ** 3 / t6)
        f[46:63] = [t3 / fro ** 3, t4 / fro ** 4, t5 / fro ** 5, t6 / fro ** 6, er4 / n, er6 / n,
                    t4 * t4 / (t6 * fro2), t3 * t3 / (t4 * fro2), t5 / (t4 * fro), np.log(er4) / ln,
                    np.log(er6) / ln, t1 * t3 / fro ** 4, t3 / (fro * np.sqrt(t4)), t5 / np.sqrt(t4 * t6),
                    t2 / fro2, t1 / fro, er4 / er6]
    f[63] = np.sort(r2)[::-1][:16].sum() / fro2
    return f
