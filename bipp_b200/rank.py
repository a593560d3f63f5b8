"""Learned rank predictor: how many eigenpairs of a time step lie above the energy
threshold, predicted from the whitened visibility matrix by a small MLP, so that the
eigensolver computes the largest k + margin eigenpairs instead of all of them (with a
fallback to the full solve). No counterpart in the reference, which computes every
eigenpair with LAPACK ?hegv (src/eigensolver.cpp:188-216).

Everything numeric runs in the library: the features and the labels come from the
method's own eigensolver (bipp_rank_features_s), the network is trained on the GPU by its
hand-written forward, backward and Adam kernels (bipp_rank_mlp_train), and the ranked
eigensolver (bipp_eigh_gram_batched_ranked_s) runs the predicted partial solve.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from ._lib import check
from .api import Context, _ptr, default_context

N_FEATURES = 64
HIDDEN = 128
MODES = {"full": 0, "exact": 1, "predicted": 2}


def num_params(ctx: Optional[Context] = None) -> int:
    ctx = ctx or default_context()
    return int(ctx._lib.bipp_rank_mlp_num_params())


def features(wl, s, xyz, threshold: float = 0.0, ctx: Optional[Context] = None):
    """(features [B, 64] float32, counts [B]) of steps s [B, N, N] (complex64, W = I),
    xyz [B, N, 3], wl [B]: the full solve's count of eigenvalues above the threshold is the
    training label."""
    ctx = ctx or default_context()
    wl = np.ascontiguousarray(wl, dtype=np.float32)
    s = np.asarray(s, dtype=np.complex64)
    B, N = s.shape[0], s.shape[1]
    sF = np.ascontiguousarray(np.transpose(s, (0, 2, 1)))
    xyzF = np.ascontiguousarray(np.transpose(np.asarray(xyz, dtype=np.float32), (0, 2, 1)))
    f = np.zeros((B, N_FEATURES), dtype=np.float32)
    counts = np.zeros(B, dtype=np.int32)
    check(ctx._lib.bipp_rank_features_s(ctx.handle, B, N, _ptr(wl), _ptr(sF), _ptr(xyzF), C.c_double(threshold),
                                        _ptr(f), _ptr(counts)))
    return f, counts


def init_model(feats, seed: int = 0, ctx: Optional[Context] = None) -> np.ndarray:
    """A fresh model: the features' mean and standard deviation, the latter at least
    1e-4 (every feature is scale free, and those that vary less across steps, such as
    the diagonal of the whitened matrix, which is tiny against its norm, are dominated by
    the FP32 rounding of that matrix and must not be magnified into noise of unit size),
    He-normal weights, zero biases."""
    feats = np.asarray(feats, dtype=np.float64)
    rng = np.random.default_rng(seed)
    mu = feats.mean(0)
    sd = np.maximum(feats.std(0), 1e-4)
    w1 = rng.standard_normal((N_FEATURES, HIDDEN)) * np.sqrt(2.0 / N_FEATURES)
    w2 = rng.standard_normal((HIDDEN, HIDDEN)) * np.sqrt(2.0 / HIDDEN)
    w3 = rng.standard_normal(HIDDEN) * np.sqrt(1.0 / HIDDEN)
    m = np.concatenate([mu, sd, w1.reshape(-1), np.zeros(HIDDEN), w2.reshape(-1), np.zeros(HIDDEN), w3, [0.0]])
    assert m.size == num_params(ctx)
    return m.astype(np.float32)


def forward(model, feats, ctx: Optional[Context] = None) -> np.ndarray:
    ctx = ctx or default_context()
    model = np.ascontiguousarray(model, dtype=np.float32)
    feats = np.ascontiguousarray(feats, dtype=np.float32)
    out = np.zeros(feats.shape[0], dtype=np.float32)
    check(ctx._lib.bipp_rank_mlp_forward(ctx.handle, _ptr(model), _ptr(feats), feats.shape[0], _ptr(out)))
    return out


def gradient(model, feats, targets, ctx: Optional[Context] = None):
    """(loss, gradient [num_params]) of the mean squared error."""
    ctx = ctx or default_context()
    model = np.ascontiguousarray(model, dtype=np.float32)
    feats = np.ascontiguousarray(feats, dtype=np.float32)
    targets = np.ascontiguousarray(targets, dtype=np.float32)
    grad = np.zeros(model.size, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    check(ctx._lib.bipp_rank_mlp_gradient(ctx.handle, _ptr(model), _ptr(feats), _ptr(targets), feats.shape[0],
                                          _ptr(grad), _ptr(loss)))
    return float(loss[0]), grad


def train(model, feats, targets, iterations: int = 2000, lr: float = 1e-3, weight_decay: float = 0.0,
          val_feats=None, val_targets=None, eval_every: int = 100, ctx: Optional[Context] = None):
    """(trained model, loss history, validation history): full-batch Adam on the GPU with
    the L2 penalty (weight_decay / 2) |W|^2 of the weights; with a validation set the
    model of lowest validation loss is returned."""
    ctx = ctx or default_context()
    model = np.array(model, dtype=np.float32, copy=True)
    feats = np.ascontiguousarray(feats, dtype=np.float32)
    targets = np.ascontiguousarray(targets, dtype=np.float32)
    hist = np.zeros(iterations, dtype=np.float32)
    nv = 0 if val_feats is None else len(val_feats)
    vf = np.ascontiguousarray(val_feats, dtype=np.float32) if nv else None
    vt = np.ascontiguousarray(val_targets, dtype=np.float32) if nv else None
    vh = np.zeros(max(1, -(-iterations // eval_every)), dtype=np.float32)
    check(ctx._lib.bipp_rank_mlp_train(ctx.handle, _ptr(model), _ptr(feats), _ptr(targets), feats.shape[0],
                                       _ptr(vf) if nv else None, _ptr(vt) if nv else None, nv, int(iterations),
                                       C.c_float(lr), C.c_float(weight_decay), int(eval_every), _ptr(hist), _ptr(vh)))
    return model, hist, (vh if nv else None)


def eigh_gram_ranked(wl, s, xyz, threshold: float = 0.0, mode: str = "predicted", model=None, margin: int = 16,
                     residual_tol: float = -1.0, ctx: Optional[Context] = None, vectors: bool = True):
    """Ranked batched eigh_gram (W = I): mode "full" (every eigenpair), "exact" (those
    above the threshold, exact range) or "predicted" (largest k + margin, k from the
    model, fallback to full). Returns dict(v, d, nred, scale, k_computed, fallback, ms)."""
    ctx = ctx or default_context()
    wl = np.ascontiguousarray(wl, dtype=np.float32)
    s = np.asarray(s, dtype=np.complex64)
    B, N = s.shape[0], s.shape[1]
    sF = np.ascontiguousarray(np.transpose(s, (0, 2, 1)))
    xyzF = np.ascontiguousarray(np.transpose(np.asarray(xyz, dtype=np.float32), (0, 2, 1)))
    d = np.zeros((B, N), dtype=np.float32)
    vF = np.zeros((B, N, N), dtype=np.complex64) if vectors else None
    nred = np.zeros(B, dtype=np.uint64)
    scale = np.zeros(B, dtype=np.float32)
    kc = np.zeros(B, dtype=np.int32)
    fb = np.zeros(B, dtype=np.int32)
    ms = C.c_double()
    m = np.ascontiguousarray(model, dtype=np.float32) if model is not None else None
    check(ctx._lib.bipp_eigh_gram_batched_ranked_s(
        ctx.handle, B, N, _ptr(wl), _ptr(sF), _ptr(xyzF), C.c_double(threshold), MODES[mode],
        _ptr(m) if m is not None else None, int(margin), C.c_double(residual_tol), _ptr(d),
        _ptr(vF) if vF is not None else None, _ptr(nred), _ptr(scale), _ptr(kc), _ptr(fb), C.byref(ms)))
    v = np.transpose(vF, (0, 2, 1)) if vF is not None else None
    return {"v": v, "d": d, "nred": nred.astype(np.int64), "scale": scale, "k_computed": kc, "fallback": fb,
            "ms": ms.value}


def c4_steps(obs, steps, chunk: int = 512):
    """Host arrays (s, xyz, wl) of rank-predictor workload steps, generated on the GPU."""
    import torch

    from . import simulate as sim

    dev = torch.device("cuda", torch.cuda.current_device())
    S, X = [], []
    for i0 in range(0, len(steps), chunk):
        s, x = sim.visibilities_c4(obs, steps[i0:i0 + chunk], device=dev)
        S.append(s.cpu().numpy())
        X.append(x.cpu().numpy())
    s, x = np.concatenate(S), np.concatenate(X)
    return s, x, np.full(len(steps), obs.cfg.wl, dtype=np.float32)


def study(ctx, obs, n_train: int = 2000, n_eval: int = 2000, threshold: float = 0.0, iterations: int = 3000,
          lr: float = 1e-3, margin: int = 16, seed: int = 0, chunk: int = 512, weight_decay: float = 1e-3):
    """The rank-predictor study on the workload of `obs` (config_c4): train on the first
    n_train steps (features and labels from the full solve; the last fifth of them
    validates, and the model of lowest validation loss is kept), then solve the next n_eval
    steps in the three modes, chunk steps per call. Reports the loss, the fallback rate, the
    count error of the prediction, the eigenvalue error of the predicted partial solve
    against the full solve (eigenvalues above the threshold), and the eigensolver device
    time of each mode."""
    s, x, wl = c4_steps(obs, list(range(n_train)))
    feats, counts = features(wl, s, x, threshold, ctx=ctx)
    nred = np.count_nonzero(np.abs(s).sum(1) > 0, axis=1)
    y = counts / np.maximum(nred, 1)
    # the last fifth of the training steps is the validation set of the early stopping
    nt = n_train - n_train // 5
    model, hist, vhist = train(init_model(feats[:nt], seed, ctx=ctx), feats[:nt], y[:nt], iterations=iterations,
                               lr=lr, weight_decay=weight_decay, val_feats=feats[nt:], val_targets=y[nt:],
                               eval_every=100, ctx=ctx)
    se, xe, wle = c4_steps(obs, list(range(n_train, n_train + n_eval)))
    res = {m: [] for m in MODES}
    for i0 in range(0, n_eval, chunk):
        sl = slice(i0, min(n_eval, i0 + chunk))
        for m in MODES:
            res[m].append(eigh_gram_ranked(wle[sl], se[sl], xe[sl], threshold, m, model if m == "predicted" else None,
                                           margin, ctx=ctx, vectors=False))
    cat = {m: {k: np.concatenate([r[k] for r in res[m]]) for k in ("d", "k_computed", "fallback")} for m in MODES}
    ms = {m: float(sum(r["ms"] for r in res[m])) for m in MODES}
    d_full, d_pred = cat["full"]["d"], cat["predicted"]["d"]
    above = d_full > threshold
    scale = np.abs(d_full).max(1, keepdims=True)
    err = np.abs(np.where(above, d_pred - d_full, 0.0)) / np.maximum(scale, 1e-30)
    k_true = above.sum(1)
    feats_e, _ = features(wle, se, xe, threshold, ctx=ctx)
    nred_e = np.count_nonzero(np.abs(se).sum(1) > 0, axis=1)
    k_pred = np.clip(np.rint(forward(model, feats_e, ctx=ctx) * nred_e), 0, nred_e).astype(int)
    return {
        "train_steps": n_train, "eval_steps": n_eval, "threshold": threshold, "margin": margin,
        "loss_first": float(hist[0]), "loss_last": float(hist[-1]), "val_loss_best": float(vhist.min()),
        "fallback_rate": float(cat["predicted"]["fallback"].mean()),
        "count_error_mean_abs": float(np.abs(k_pred - k_true).mean()),
        "count_error_max_under": int(max(0, (k_true - k_pred).max())),
        "eig_err_vs_full_normwise": float(err.max()),
        "vectors_per_step": {m: float(cat[m]["k_computed"].mean()) for m in MODES},
        "eigensolver_ms": ms,
        "steps_per_s": {m: n_eval / (ms[m] / 1000.0) for m in MODES},
        "model": model,
    }
