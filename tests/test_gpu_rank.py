"""GPU: the learned rank predictor (bipp_b200.rank): features of the whitened matrix,
the MLP's forward pass, gradient and Adam training on the device against the numpy
oracle (oracle/mlp.py), and the predicted partial solve with its fallback against the
full solve and the exact (Sturm-count) range solve on the rank-predictor workload
(256 antennas in a 10 km disc, 5-200 sources and a noise level per step).

Tolerances: forward pass 1e-5 relative, gradient 1e-4 of its largest component, features
1e-4 against numpy on the FP64 whitened matrix; eigenvalues of the partial solve equal to
the full solve's above the threshold (same bisection), V diag(d) V^H to 1e-5."""
import numpy as np
import pytest

from oracle import mlp as om

pytestmark = pytest.mark.gpu


def _random_model(seed=0, n=300):
    from bipp_b200 import rank

    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((n, 64)) * rng.uniform(0.1, 3.0, 64) + rng.uniform(-1, 1, 64)).astype(np.float32)
    model = rank.init_model(X, seed)
    model[om.OFF["b1"]:om.OFF["W2"]] = rng.uniform(-0.1, 0.1, 128)   # nonzero biases
    model[om.OFF["b2"]:om.OFF["W3"]] = rng.uniform(-0.1, 0.1, 128)
    model[om.OFF["b3"]] = 0.25
    y = rng.uniform(0, 1, n).astype(np.float32)
    return model, X, y


def test_mlp_forward_and_gradient_against_oracle(ctx):
    from bipp_b200 import rank

    assert rank.num_params(ctx) == om.N_PARAMS
    model, X, y = _random_model(1, n=301)   # not a multiple of the 16-sample tile
    out = rank.forward(model, X, ctx=ctx)
    ref, _ = om.forward(model, X)
    assert np.abs(out - ref).max() <= 1e-5 * np.abs(ref).max()
    loss, g = rank.gradient(model, X, y, ctx=ctx)
    lref, gref = om.loss_and_gradient(model, X, y)
    assert abs(loss - lref) <= 1e-5 * lref
    assert np.all(g[:om.OFF["W1"]] == 0)
    assert np.abs(g - gref).max() <= 1e-4 * np.abs(gref).max(), np.abs(g - gref).max() / np.abs(gref).max()


def test_mlp_adam_step_and_training(ctx):
    """One training iteration is one Adam step on the GPU gradient (first step: -lr g /
    (|g| + eps)); a longer run fits a smooth function of the features."""
    from bipp_b200 import rank

    model, X, _ = _random_model(2, n=512)
    y = (0.4 + 0.2 * np.tanh(X[:, 0] / 3) - 0.1 * np.tanh(X[:, 5] * X[:, 9] / 4)).astype(np.float32)
    _, g = rank.gradient(model, X, y, ctx=ctx)
    m1, h1, _ = rank.train(model, X, y, iterations=1, lr=1e-3, ctx=ctx)
    step = m1.astype(np.float64) - model
    expect = -1e-3 * g / (np.abs(g) + 1e-8)
    big = np.abs(g) > 1e-5
    assert np.all(step[:om.OFF["W1"]] == 0)
    assert np.abs(step[big] - expect[big]).max() <= 2e-6
    trained, hist, _ = rank.train(model, X, y, iterations=1500, lr=2e-3, ctx=ctx)
    print(f"loss {hist[0]:.4f} -> {hist[-1]:.5f}")
    assert hist[-1] <= 0.05 * hist[0]
    lfin, _ = om.loss_and_gradient(trained, X, y)
    assert lfin <= 0.05 * hist[0]


def test_training_keeps_the_best_validation_model(ctx):
    """With a validation set the returned model is the one of lowest validation loss
    (checked with the numpy oracle), and weight decay shrinks the weights."""
    from bipp_b200 import rank

    model, X, _ = _random_model(4, n=400)
    y = (0.5 + 0.3 * np.tanh(X[:, 1] / 2)).astype(np.float32)
    Xv, yv = X[300:], y[300:]
    trained, hist, vh = rank.train(model, X[:300], y[:300], iterations=600, lr=2e-3, val_feats=Xv,
                                   val_targets=yv, eval_every=50, ctx=ctx)
    lv, _ = om.loss_and_gradient(trained, Xv, yv)
    assert abs(lv - vh.min()) <= 1e-4 * max(vh.min(), 1e-6) + 1e-7
    plain, _, _ = rank.train(model, X[:300], y[:300], iterations=300, lr=2e-3, ctx=ctx)
    decayed, _, _ = rank.train(model, X[:300], y[:300], iterations=300, lr=2e-3, weight_decay=0.5, ctx=ctx)
    w = slice(om.OFF["W1"], om.N_PARAMS)
    assert np.linalg.norm(decayed[w]) < np.linalg.norm(plain[w])


def test_features_against_numpy_whitened_matrix(ctx):
    """Features of the GPU against the numpy statement on the FP64 whitened matrix
    L^-1 S L^-H (oracle Gram matrix and Cholesky)."""
    import scipy.linalg as sla

    from bipp_b200 import rank
    from bipp_b200 import simulate as sim
    from oracle import bluebild as bb

    cfg = sim.config_c4()
    obs = sim.observation(cfg)
    s, x = sim.visibilities_c4(obs, [3, 4, 5])
    s, x = s.numpy(), x.numpy()
    wl = np.full(3, cfg.wl, dtype=np.float32)
    f, counts = rank.features(wl, s, x, 0.0, ctx=ctx)
    for k in range(3):
        G = bb.gram_matrix(np.eye(cfg.n_antenna), x[k].astype(np.float32).astype(np.float64), float(wl[k]))
        L = np.linalg.cholesky(G)
        Li = sla.solve_triangular(L, np.eye(cfg.n_antenna), lower=True)
        Cw = Li @ s[k].astype(np.complex128) @ Li.conj().T
        fr = om.features(Cw, 0.0)
        assert np.abs(f[k] - fr).max() <= 1e-4 * max(1.0, np.abs(fr).max()), np.abs(f[k] - fr).max()
        d = np.linalg.eigvalsh(Cw)
        assert abs(counts[k] - np.count_nonzero(d > 0)) <= 1


def _vv(v, d, thr):
    sel = d > thr
    vs = v[:, sel].astype(np.complex128)
    return (vs * d[sel]) @ vs.conj().T


def test_predicted_partial_solve_study(ctx):
    """Train on 2000 method-generated steps, solve 512 others: the predicted partial
    solve (k + 16 eigenpairs, fallback to full) returns the full solve's eigenvalues above
    the threshold and computes fewer eigenvectors than the full solve; the device times
    of the three modes (full, exact Sturm-count range, predicted) are printed, not
    asserted, as the features cost about what the skipped eigenvectors save at 256
    antennas."""
    from bipp_b200 import rank
    from bipp_b200 import simulate as sim

    obs = sim.observation(sim.config_c4())
    r = rank.study(ctx, obs, n_train=2000, n_eval=512, iterations=3000, lr=1e-3)
    r.pop("model")
    print(r)
    assert r["loss_last"] < 0.2 * r["loss_first"]
    assert r["eig_err_vs_full_normwise"] <= 1e-6
    assert r["fallback_rate"] <= 0.1
    v = r["vectors_per_step"]
    assert v["predicted"] < v["full"] and v["exact"] <= v["predicted"]


def test_partial_solve_fallbacks_give_the_full_solve(ctx):
    """Both fallbacks: a model that predicts no eigenvalue above the threshold (the last
    Ritz value is then above it) and a residual tolerance of 0 (every residual check
    fails) make every step fall back; eigenvalues and V diag(d) V^H above the threshold
    equal the full solve's."""
    from bipp_b200 import rank
    from bipp_b200 import simulate as sim

    cfg = sim.config_c4()
    obs = sim.observation(cfg)
    s, x, wl = rank.c4_steps(obs, list(range(100, 140)))
    full = rank.eigh_gram_ranked(wl, s, x, 0.0, "full", ctx=ctx)
    exact = rank.eigh_gram_ranked(wl, s, x, 0.0, "exact", ctx=ctx)
    feats, counts = rank.features(wl, s, x, 0.0, ctx=ctx)
    model = rank.init_model(feats, 0)
    model[om.OFF["W3"]:] = 0.0
    model[om.OFF["b3"]] = -1.0                       # predicts k = 0
    low = rank.eigh_gram_ranked(wl, s, x, 0.0, "predicted", model, margin=2, ctx=ctx)
    model[om.OFF["b3"]] = 2.0                        # predicts k = n (full range, no fallback)
    every = rank.eigh_gram_ranked(wl, s, x, 0.0, "predicted", model, ctx=ctx)
    model[om.OFF["b3"]] = 0.5
    res = rank.eigh_gram_ranked(wl, s, x, 0.0, "predicted", model, residual_tol=0.0, ctx=ctx)
    assert np.all(low["fallback"][counts > 2] == 1)
    assert np.all(every["fallback"] == 0)
    assert np.all(res["fallback"] == 1)
    n = full["nred"]
    assert np.all(full["k_computed"] == n)
    assert np.all(low["k_computed"][low["fallback"] == 1] == n[low["fallback"] == 1])
    assert np.all(every["k_computed"] == n) and np.all(res["k_computed"] == n)
    for k in range(len(wl)):
        above = full["d"][k] > 0
        for out in (low, every, res, exact):
            assert np.abs(out["d"][k][above] - full["d"][k][above]).max() <= 1e-6 * np.abs(full["d"][k]).max()
            p, pf = _vv(out["v"][k], out["d"][k], 0.0), _vv(full["v"][k], full["d"][k], 0.0)
            assert np.abs(p - pf).max() <= 1e-5 * np.abs(pf).max()
