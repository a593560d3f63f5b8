"""GPU: the autotuner of launch shapes (bipp_autotune_pipeline). It times every candidate
of the tunable parameters on a sample batch, keeps the fastest in the tuning table,
leaves the pipeline's images untouched, and the images computed with the tuned values
agree with those of the defaults (1e-5 relative L2 per level; only the summation order
of the spreading and the tridiagonalisation changes)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_pipeline(ctx):
    import torch

    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim
    from bipp_b200.parameter_estimator import infer_intervals

    bipp.tuning_reset()
    cfg = sim.config_c2(n_antenna=256, n_steps=64, image_size=256, n_src=100, keep=(200, 256))
    obs = sim.observation(cfg)
    dev = torch.device("cuda", 0)
    s, x = sim.visibilities(obs, list(range(64)), device=dev, dtype=torch.complex64, masks=sim.keep_masks(cfg))
    S = s.transpose(1, 2).contiguous()
    wl = torch.full((64,), cfg.wl, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    _, d, _, _ = bipp.eigh_gram_batched(np.full(8, cfg.wl, np.float32), s[:8].cpu().numpy(), x[:8].cpu().numpy(),
                                        ctx=ctx)
    intervals = infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, d)
    n = cfg.image_size
    l = obs.lmn[:, 0].reshape(n, n)
    m = obs.lmn[:, 1].reshape(n, n)
    lat = (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, lat, obs.lmn[:, 2], obs.basis, tolerance=cfg.eps,
                       chunk_steps=64, max_steps=64)
    pl.process_device(64, S.data_ptr(), x.data_ptr(), wl.data_ptr())
    base = pl.images().astype(np.float64)
    names = ("spread.items_cap", "spread.operands", "spread.stages", "spread.ctas_per_sm", "spread.schedule",
             "hetrd.threads", "hetrd.ctas_pct", "tridiag.threads", "vv.ctas_per_sm")
    start = {name: bipp.tuning_get(name) for name in names}
    rep = pl.autotune(64, S.data_ptr(), x.data_ptr(), wl.data_ptr(), on_device=True, repeats=1)
    print(rep)
    desc = bipp.tuning_describe()
    whole = rep["whole_call_ms"]
    assert whole["kept"] in ("tuned", "starting")
    assert (whole["tuned"] <= whole["starting"]) == (whole["kept"] == "tuned")
    for name in names:
        # the tuned values, or the starting ones if the tuned set made the whole call slower
        assert desc[name]["value"] == (rep[name]["chosen"] if whole["kept"] == "tuned" else start[name])
        assert sorted(int(k) for k in rep[name] if k != "chosen") == desc[name]["candidates"]
    assert np.array_equal(pl.images().astype(np.float64), base)   # images left as they were
    pl.reset()
    pl.process_device(64, S.data_ptr(), x.data_ptr(), wl.data_ptr())
    tuned = pl.images().astype(np.float64)
    for lv in range(tuned.shape[0]):
        assert np.linalg.norm(tuned[lv] - base[lv]) <= 1e-5 * np.linalg.norm(base[lv]), lv
    pl.close()
    bipp.tuning_reset()


def test_spreader_variants_agree(ctx):
    """The tunable spreader variants (one or two operand stages; tf32-split operands with
    A in shared or tensor memory, or FP16 hi/lo operands; round-robin or heaviest-first
    dynamic schedule; work-item caps) give the same images to 1e-5
    relative L2 per level on a batch that splits heavy tiles (the cap changes which tiles
    are split, so the FP32 sums of their parts are added in another order: differences of
    ~2e-6 were measured)."""
    import torch

    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim
    from bipp_b200.parameter_estimator import infer_intervals

    bipp.tuning_reset()
    cfg = sim.config_c2(n_antenna=256, n_steps=96, image_size=256, n_src=100, keep=(200, 256))
    obs = sim.observation(cfg)
    dev = torch.device("cuda", 0)
    s, x = sim.visibilities(obs, list(range(96)), device=dev, dtype=torch.complex64, masks=sim.keep_masks(cfg))
    S = s.transpose(1, 2).contiguous()
    wl = torch.full((96,), cfg.wl, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    _, d, _, _ = bipp.eigh_gram_batched(np.full(8, cfg.wl, np.float32), s[:8].cpu().numpy(), x[:8].cpu().numpy(),
                                        ctx=ctx)
    intervals = infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, d)
    n = cfg.image_size
    l = obs.lmn[:, 0].reshape(n, n)
    m = obs.lmn[:, 1].reshape(n, n)
    lat = (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, lat, obs.lmn[:, 2], obs.basis, tolerance=cfg.eps,
                       chunk_steps=96, max_steps=96)

    def run():
        pl.reset()
        pl.process_device(96, S.data_ptr(), x.data_ptr(), wl.data_ptr())
        return pl.images().astype(np.float64), pl.nufft_stats()

    base, st = run()
    assert st["split_tiles"] > 0 or bipp.tuning_get("spread.items_cap") > 2048
    for settings in ({"spread.stages": 1}, {"spread.schedule": 0}, {"spread.items_cap": 8192},
                     {"spread.operands": 0, "spread.stages": 1},
                     {"spread.operands": 0, "spread.stages": 2, "spread.schedule": 0},
                     {"spread.operands": 1, "spread.stages": 1}, {"spread.operands": 1, "spread.stages": 2}):
        bipp.tuning_reset()
        for k, v in settings.items():
            bipp.tuning_set(k, v)
        got, _ = run()
        for lv in range(got.shape[0]):
            assert np.linalg.norm(got[lv] - base[lv]) <= 1e-5 * np.linalg.norm(base[lv]), (settings, lv)
    bipp.tuning_reset()
    pl.close()


def test_persistent_tridiagonalisation_agrees(ctx):
    """The eigensolver's tunable launch shapes give the eigenvalues and V diag(d) V^H of
    the defaults, to 1e-6 relative, on 40 steps of uneven size (100-160 of 160 antennas
    kept, so that the blocked panels run): the tridiagonalisation as persistent CTAs
    (fewer than the matrices, each taking matrices in the size order) and the
    back-transform on 32-column slices."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    bipp.tuning_reset()
    cfg = sim.config_c2(n_antenna=160, n_steps=40, image_size=64, n_src=20, keep=(100, 160))
    obs = sim.observation(cfg)
    s, x = sim.visibilities(obs, list(range(40)), masks=sim.keep_masks(cfg))
    s, x = s.numpy().astype(np.complex64), x.numpy().astype(np.float32)
    wl = np.full(40, cfg.wl, np.float32)
    v0, d0, n0, _ = bipp.eigh_gram_batched(wl, s, x, ctx=ctx)
    try:
        for pct in (("hetrd.ctas_pct", 50), ("hetrd.ctas_pct", 150), ("bt.columns", 32), ("tridiag.threads", 128)):
            bipp.tuning_reset()
            bipp.tuning_set(*pct)
            v1, d1, n1, _ = bipp.eigh_gram_batched(wl, s, x, ctx=ctx)
            assert np.array_equal(n0, n1)
            for b in range(40):
                sc = np.abs(d0[b]).max()
                assert np.abs(d1[b] - d0[b]).max() <= 1e-6 * sc, (pct, b)
                k = int(n0[b])
                a0 = (v0[b][:, :k] * d0[b][:k]) @ v0[b][:, :k].conj().T
                a1 = (v1[b][:, :k] * d1[b][:k]) @ v1[b][:, :k].conj().T
                assert np.linalg.norm(a1 - a0) <= 1e-6 * np.linalg.norm(a0), (pct, b)
    finally:
        bipp.tuning_reset()
