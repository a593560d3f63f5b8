"""GPU parity of the synthesis path: direct nuft_sum, partition, collect/get NUFFT,
dataset-driven image_synthesis and the batched pipeline, against the FP64 oracle
(direct sums in FP64) and the reference's own outputs.

Tolerances: direct sum FP32 entry 1e-5 relative (max-norm), FP64 entry 1e-10; NUFFT
images 1e-4 relative L2 at tolerance 1e-5 (10 x eps + FP32 accumulation); pipeline
image stack 1e-4 relative L2 against the FP64 oracle."""
import math

import numpy as np
import pytest

from conftest import golden
from oracle import bluebild as bb

pytestmark = pytest.mark.gpu


def _rel_l2(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300)


def test_nuft_sum_f64_matches_reference(ctx):
    import bipp_b200 as bipp

    g = golden("nuft.npz")
    out = bipp.nuft_sum(float(g["alpha"]), g["vals"], g["u"], g["v"], g["w"], g["x"], g["y"], g["z"], ctx=ctx)
    assert np.abs(out - g["out64"]).max() <= 1e-10 * np.abs(g["out64"]).max()


def test_nuft_sum_f32_accumulates(ctx):
    import bipp_b200 as bipp

    g = golden("nuft.npz")
    out0 = np.full(g["x"].shape[0], 3.0, dtype=np.float32)
    out = bipp.nuft_sum(np.float32(g["alpha"]), g["vals"].astype(np.complex64), g["u"], g["v"], g["w"], g["x"],
                        g["y"], g["z"], out=out0.copy(), ctx=ctx)
    # reference float input rounding: compare against the FP64 sum of the float inputs
    f = lambda a: np.asarray(a, np.float32).astype(np.float64)  # noqa: E731
    exact = bb.nuft_sum(float(np.float32(g["alpha"])), g["vals"].astype(np.complex64), f(g["u"]), f(g["v"]), f(g["w"]),
                        f(g["x"]), f(g["y"]), f(g["z"]))
    assert np.abs(out - 3.0 - exact).max() <= 1e-5 * np.abs(exact).max()


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("n", [1, 100, 4000])
def test_partition_matches_reference(ctx, n, prec):
    import bipp_b200 as bipp

    g = golden("partition.npz")
    pm, gb, gs = bipp.domain_partition_grid([2, 3, 4], g[f"x_{n}_{prec}"], g[f"y_{n}_{prec}"], g[f"z_{n}_{prec}"],
                                            ctx=ctx)
    assert (pm == g[f"permut_{n}_{prec}"]).all()
    assert (gb == g[f"begin_{n}_{prec}"]).all()
    assert (gs == g[f"size_{n}_{prec}"]).all()


def test_partition_single_point_and_identity(ctx):
    import bipp_b200 as bipp

    pm, gb, gs = bipp.domain_partition_grid([2, 3, 4], [1.0], [2.0], [3.0], ctx=ctx)
    assert list(pm) == [0] and gs.sum() == 1
    pm, gb, gs = bipp.domain_partition_grid([1, 1, 1], np.arange(5.0), np.arange(5.0), np.arange(5.0), ctx=ctx)
    assert list(pm) == list(range(5)) and list(gs) == [5]


def _synthetic_points(rng, m, umax, wmax):
    u, v = rng.uniform(-umax, umax, (2, m))
    w = rng.uniform(-wmax, wmax, m)
    c = rng.standard_normal((m, 2)) + 1j * rng.standard_normal((m, 2))
    return np.stack([u, v, w], 1), c


@pytest.mark.parametrize("tol", [1e-3, 1e-5, 1e-7])
def test_nufft_collect_get_lattice(ctx, tol):
    """Collect/get NUFFT on a make_grids pixel lattice (float lmn, first-order residual
    channels active) against the FP64 direct sum of the same float inputs."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    rng = np.random.default_rng(5)
    lmn = sim.make_lmn_grid(48, math.radians(12.0)).astype(np.float32)
    opt = bipp.NufftSynthesisOptions().set_tolerance(tol)
    nb = 700
    plan = bipp.NufftSynthesis(ctx, opt, lmn, 2, nb)
    pts = []
    for _ in range(3):
        uvw, c = _synthetic_points(rng, nb, 4000.0, 300.0)
        uvw = uvw.astype(np.float32)
        c = c.astype(np.complex64)
        plan.add(uvw, c)
        pts.append((uvw, c))
    imgs = [plan.get_image(i) for i in range(2)]
    uvw = np.concatenate([p[0] for p in pts]).astype(np.float64)
    c = np.concatenate([p[1] for p in pts]).astype(np.complex128)
    l64 = lmn.astype(np.float64)
    for i in range(2):
        ref_img = bb.nuft_sum(1.0, c[:, i], uvw[:, 0], uvw[:, 1], uvw[:, 2], l64[:, 0], l64[:, 1], l64[:, 2])
        assert _rel_l2(imgs[i], ref_img) <= max(20 * tol, 2e-6)
    plan.close()


@pytest.mark.parametrize("na,nb_", [(40, 64), (16, 1024), (24, 432)])
def test_pruned_fft_rectangular_lattice(ctx, na, nb_):
    """Rectangular pixel lattices whose fine grids take different pruned-FFT plans for the
    rows (along x) and the columns (along y): 40 x 64 px -> 80 x 112 cells (rows
    112 = 7 x 16, columns 80 = 5 x 16), 16 x 1024 px -> 32 x 1792 (rows 7 x 16 x 16 with
    the block shared-memory layout, the 1024^2-pixel workload's row length; columns 8 x 4),
    24 x 432 px -> 48 x 768 (rows 3 x 16 x 16, columns 3 x 16). Each images like the FP64
    direct sum with the pruned transform and with the full 2-D cuFFT transform
    (nufft.fft = 0); the two differ in their rounding only, so the pruned kernels, not a
    fallback, ran."""
    import bipp_b200 as bipp

    rng = np.random.default_rng(17)
    a, b = np.meshgrid(np.arange(na), np.arange(nb_), indexing="ij")
    l = (b.reshape(-1) - nb_ / 2 + 0.5) * (0.2 / nb_)
    m = (a.reshape(-1) - na / 2 + 0.25) * (0.11 / na)
    lmn = np.stack([l, m, np.sqrt(1 - l * l - m * m)], 1).astype(np.float32)
    npts = 900
    pts = [_synthetic_points(rng, npts, 700.0, 60.0) for _ in range(2)]
    uvw = np.concatenate([p[0] for p in pts]).astype(np.float32).astype(np.float64)
    c = np.concatenate([p[1] for p in pts]).astype(np.complex64).astype(np.complex128)
    l64 = lmn.astype(np.float64)
    imgs = {}
    try:
        for fft in (1, 0):
            bipp.tuning_set("nufft.fft", fft)
            plan = bipp.NufftSynthesis(ctx, bipp.NufftSynthesisOptions().set_tolerance(1e-7), lmn, 2, npts)
            for u, v in pts:
                plan.add(u.astype(np.float32), v.astype(np.complex64))
            imgs[fft] = [plan.get_image(i) for i in range(2)]
            plan.close()
    finally:
        bipp.tuning_reset()
    for i in range(2):
        ref_img = bb.nuft_sum(1.0, c[:, i], uvw[:, 0], uvw[:, 1], uvw[:, 2], l64[:, 0], l64[:, 1], l64[:, 2])
        for fft in (0, 1):
            assert _rel_l2(imgs[fft][i], ref_img) <= 2e-6, (fft, i)
        assert _rel_l2(imgs[1][i], imgs[0][i]) <= 1e-6
        assert not np.array_equal(imgs[1][i], imgs[0][i])


def test_nufft_collect_get_four_images_warp_spreader(ctx):
    """Four images on a make_grids lattice with the first-order residual channels active:
    12 channels, more than the tensor-core spreader takes, so the warp spreader with
    shared-memory atomics runs; against the FP64 direct sum of the same float inputs."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    rng = np.random.default_rng(9)
    lmn = sim.make_lmn_grid(48, math.radians(12.0)).astype(np.float32)
    tol = 1e-5
    plan = bipp.NufftSynthesis(ctx, bipp.NufftSynthesisOptions().set_tolerance(tol), lmn, 4, 600)
    pts = []
    for _ in range(3):
        u, v = rng.uniform(-4000.0, 4000.0, (2, 600))
        w = rng.uniform(-300.0, 300.0, 600)
        uvw = np.stack([u, v, w], 1).astype(np.float32)
        c = (rng.standard_normal((600, 4)) + 1j * rng.standard_normal((600, 4))).astype(np.complex64)
        plan.add(uvw, c)
        pts.append((uvw, c))
    imgs = [plan.get_image(i) for i in range(4)]
    uvw = np.concatenate([p[0] for p in pts]).astype(np.float64)
    c = np.concatenate([p[1] for p in pts]).astype(np.complex128)
    l64 = lmn.astype(np.float64)
    for i in range(4):
        ref_img = bb.nuft_sum(1.0, c[:, i], uvw[:, 0], uvw[:, 1], uvw[:, 2], l64[:, 0], l64[:, 1], l64[:, 2])
        assert _rel_l2(imgs[i], ref_img) <= 20 * tol, i
    plan.close()


def test_context_destroyed_before_its_collector():
    """A context destroyed before the NUFFT collector created on it stays alive until the
    collector is destroyed: the collector still adds, returns its image (that of a
    collector on a live context, to 1e-6) and is destroyed without error."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    rng = np.random.default_rng(8)
    lmn = sim.make_lmn_grid(32, math.radians(10.0)).astype(np.float32)
    uvw, c = _synthetic_points(rng, 300, 3000.0, 200.0)
    uvw, c = uvw.astype(np.float32), c.astype(np.complex64)
    imgs = []
    for early in (False, True):
        own = bipp.Context("GPU")
        plan = bipp.NufftSynthesis(own, bipp.NufftSynthesisOptions().set_tolerance(1e-5), lmn, 2, 300)
        if early:
            own.close()
        plan.add(uvw, c)
        imgs.append(plan.get_image(0))
        plan.close()
        own.close()
    assert _rel_l2(imgs[1], imgs[0]) <= 1e-6


def test_nufft_collect_get_non_lattice(ctx):
    """Pixels that are not on a lattice use the direct FP64 evaluation."""
    import bipp_b200 as bipp

    rng = np.random.default_rng(6)
    p = 300
    l, m = rng.uniform(-0.1, 0.1, (2, p))
    lmn = np.stack([l, m, np.sqrt(1 - l * l - m * m)], 1).astype(np.float32)
    plan = bipp.NufftSynthesis(ctx, bipp.NufftSynthesisOptions().set_tolerance(1e-6), lmn, 1, 400)
    uvw, c = _synthetic_points(rng, 400, 2000.0, 100.0)
    plan.add(uvw.astype(np.float32), c[:, :1].astype(np.complex64))
    img = plan.get_image(0)
    f = uvw.astype(np.float32).astype(np.float64)
    l64 = lmn.astype(np.float64)
    ref_img = bb.nuft_sum(1.0, c[:, 0].astype(np.complex64), f[:, 0], f[:, 1], f[:, 2], l64[:, 0], l64[:, 1], l64[:, 2])
    assert _rel_l2(img, ref_img) <= 1e-6


def _c1_dataset(n_steps=4, n_ant=40, image=32):
    """Small plain-Bluebild case: eigh_gram per step by the oracle, dataset in memory."""
    from bipp_b200 import simulate as sim

    cfg = sim.config_c1(n_steps=n_steps, n_antenna=n_ant, image_size=image)
    obs = sim.observation(cfg)
    s, xyz = sim.visibilities(obs, list(range(n_steps)))
    s, xyz = s.numpy(), xyz.numpy()
    steps = []
    for k in range(n_steps):
        v, d, nr, sc = bb.eigh_gram(cfg.wl, s[k], np.eye(n_ant), xyz[k], dtype=np.float32)
        steps.append(dict(v=v.astype(np.complex64), d=d.astype(np.float32), scale=sc, wl=cfg.wl,
                          uvw=sim.baseline_uvw(obs, xyz[k])))
    return cfg, obs, steps


def test_image_synthesis_dataset(ctx):
    """image_synthesis over an in-memory dataset against the FP64 oracle
    (virtual_vis + direct sum + normalisation)."""
    import bipp_b200 as bipp

    cfg, obs, steps = _c1_dataset()
    ds = bipp.InMemoryDataset(cfg.n_antenna, cfg.n_antenna)
    for k, st in enumerate(steps):
        ds.write(k, st["wl"], st["scale"], st["v"], st["d"], st["uvw"])
    dpos = [st["d"] for st in steps]
    thr = float(np.median(np.concatenate([d[d > 0] for d in dpos])))
    intervals = np.array([[0.0, thr], [thr, np.finfo(np.float32).max]])
    selection = {}
    for lv, (lo, hi) in enumerate(intervals):
        selection[f"lvl{lv}"] = {k: (st["d"] * ((st["d"] >= lo) & (st["d"] <= hi))).astype(np.float32)
                                 for k, st in enumerate(steps)}
    opt = bipp.NufftSynthesisOptions().set_tolerance(1e-6)
    out = bipp.image_synthesis(ctx, opt, ds, selection, obs.lmn.astype(np.float32))
    lmn32 = obs.lmn.astype(np.float32).astype(np.float64)
    oracle_img = bb.image_synthesis(
        [dict(uvw=st["uvw"], v=st["v"], d=st["d"], scale=st["scale"], wl=np.float32(st["wl"])) for st in steps],
        intervals, lmn32)
    got = np.stack([out["lvl0"], out["lvl1"]], 1)
    # the FP32 uvw scaling of the reference's single-precision path is part of the
    # contract; the oracle scales in FP64, so the bound includes that rounding
    assert _rel_l2(got, oracle_img) <= 2e-4


def test_image_synthesis_validation(ctx):
    import bipp_b200 as bipp

    ds = bipp.InMemoryDataset(4, 4)
    ds.write(0, 2.0, 1.0, np.eye(4), np.ones(4), np.zeros((16, 3)))
    lmn = np.zeros((4, 3), np.float32)
    opt = bipp.NufftSynthesisOptions()
    with pytest.raises(bipp.InvalidParameterError):
        bipp.image_synthesis(ctx, opt, ds, {"a/b": {0: np.ones(4)}}, lmn)
    with pytest.raises(bipp.InvalidParameterError):
        bipp.image_synthesis(ctx, opt, ds, {"a": {5: np.ones(4)}}, lmn)
    with pytest.raises(bipp.InvalidParameterError):
        bipp.image_synthesis(ctx, opt, ds, {"a": {0: np.ones(3)}}, lmn)


def _pipeline_case(n_ant=48, n_steps=6, image=40, seed=2, keep=None):
    from bipp_b200 import simulate as sim

    cfg = sim.config_c2(n_antenna=n_ant, n_steps=n_steps, image_size=image, n_src=30, seed=seed, keep=keep,
                        extent_m=8000.0)
    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    s, xyz = sim.visibilities(obs, list(range(n_steps)), masks=masks)
    return cfg, obs, s.numpy(), xyz.numpy()


def _lattice(obs, n):
    lmn = obs.lmn
    l = lmn[:, 0].reshape(n, n)
    m = lmn[:, 1].reshape(n, n)
    return (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])


def _oracle_pipeline(cfg, obs, s, xyz, intervals, filt="lsq"):
    steps = []
    for k in range(s.shape[0]):
        v, d, nr, sc = bb.eigh_gram(cfg.wl, s[k].astype(np.complex128), np.eye(cfg.n_antenna), xyz[k])
        au = xyz[k] @ obs.basis
        b = (au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3)
        steps.append(dict(uvw=b, v=v, d=d, scale=sc, wl=cfg.wl))
    # FP64 uvw (no FP32 rounding) for the pipeline oracle
    out = np.zeros((obs.lmn.shape[0], intervals.shape[0]))
    for st in steps:
        uvw = st["uvw"] * (bb.TWO_PI / st["wl"])
        for lv in range(intervals.shape[0]):
            dl = bb.level_eigenvalues(st["d"], intervals[lv, 0], intervals[lv, 1], filt)
            vv = bb.virtual_vis(st["scale"], dl, st["v"]).reshape(-1, order="F")
            out[:, lv] += bb.nuft_sum(1.0, vv, uvw[:, 0], uvw[:, 1], uvw[:, 2], obs.lmn[:, 0], obs.lmn[:, 1],
                                      obs.lmn[:, 2])
    return out / len(steps), steps


@pytest.mark.parametrize("keep", [None, (30, 48)])
def test_pipeline_batched_vs_fp64_oracle(ctx, keep):
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(keep=keep)
    d_all = np.concatenate([bb.eigh_gram(cfg.wl, s[k], np.eye(cfg.n_antenna), xyz[k])[1] for k in range(2)])
    intervals = bb.infer_intervals(3, 1.0, "log", 0.0, np.inf, d_all)
    ref_img, _ = _oracle_pipeline(cfg, obs, s, xyz, intervals)
    n = cfg.image_size
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis, tolerance=1e-6,
                       chunk_steps=4)
    pl.process(s, xyz, np.full(s.shape[0], cfg.wl))
    img = pl.images()
    err = _rel_l2(img.T, ref_img)
    assert err <= 1e-4, err
    # each level separately is close as well (bright levels tightest)
    for lv in range(intervals.shape[0]):
        assert _rel_l2(img[lv], ref_img[:, lv]) <= 5e-3
    pl.close()


@pytest.mark.parametrize("n_levels", [6, 8])
def test_pipeline_many_levels_vs_fp64_oracle(ctx, n_levels):
    """More than 4 energy levels (the 8-channel tensor-core spreader)."""
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(n_ant=48, n_steps=4, image=40)
    d_all = np.concatenate([bb.eigh_gram(cfg.wl, s[k], np.eye(cfg.n_antenna), xyz[k])[1] for k in range(2)])
    intervals = bb.infer_intervals(n_levels, 1.0, "log", 0.0, np.inf, d_all)
    ref_img, _ = _oracle_pipeline(cfg, obs, s, xyz, intervals)
    n = cfg.image_size
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis, tolerance=1e-6,
                       chunk_steps=4)
    pl.process(s, xyz, np.full(s.shape[0], cfg.wl))
    img = pl.images()
    pl.close()
    assert img.shape[0] == n_levels
    assert _rel_l2(img.T, ref_img) <= 1e-4


def test_pipeline_plain_matches_batched(ctx):
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(n_ant=32, n_steps=3, image=32)
    intervals = np.array([[0.0, 1.0], [1.0, np.inf]])
    n = cfg.image_size
    imgs = []
    for mode in ("batched", "plain"):
        pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis, tolerance=1e-6,
                           mode=mode)
        pl.process(s, xyz, np.full(s.shape[0], cfg.wl))
        imgs.append(pl.images())
        pl.close()
    assert _rel_l2(imgs[1], imgs[0].astype(np.float64)) <= 1e-4


def test_pipeline_accumulates_over_calls(ctx):
    """Splitting the steps over two process() calls gives the same normalised image
    (linearity of the synthesis in the steps)."""
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(n_ant=32, n_steps=4, image=32)
    intervals = np.array([[0.0, np.inf]])
    n = cfg.image_size
    wl = np.full(4, cfg.wl)
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis, tolerance=1e-6)
    pl.process(s, xyz, wl)
    a = pl.images()
    pl.reset()
    pl.process(s[:2], xyz[:2], wl[:2])
    pl.process(s[2:], xyz[2:], wl[2:])
    b = pl.images()
    pl.close()
    assert _rel_l2(b, a.astype(np.float64)) <= 1e-5


def test_pipeline_reads_only_lower_triangle(ctx):
    """The pipeline reads (and, for host inputs, copies) only the lower triangle of each
    S: NaN above the diagonal gives the same images."""
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(n_ant=48, n_steps=3, image=32, keep=(30, 48))
    intervals = np.array([[0.0, 1.0], [1.0, np.inf]])
    n = cfg.image_size
    wl = np.full(s.shape[0], cfg.wl)
    s_upper_nan = s.copy()
    iu = np.triu_indices(cfg.n_antenna, 1)
    for k in range(s.shape[0]):
        s_upper_nan[k][iu] = np.nan
    imgs = []
    for sk in (s, s_upper_nan):
        pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis,
                           tolerance=1e-6)
        pl.process(sk, xyz, wl)
        imgs.append(pl.images())
        pl.close()
    assert np.all(np.isfinite(imgs[1]))
    assert _rel_l2(imgs[1], imgs[0].astype(np.float64)) <= 1e-6


def test_pipeline_nonfinite_visibilities(ctx):
    """Flagged antennas given as NaN rows and columns image like zero ones; a NaN in a kept
    entry of the lower triangle of one step raises EigensolverError and adds nothing to
    the images (the reference throws at that step, before its NUFFT update)."""
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(n_ant=48, n_steps=3, image=32, keep=(30, 48))
    intervals = np.array([[0.0, 1.0], [1.0, np.inf]])
    n = cfg.image_size
    wl = np.full(s.shape[0], cfg.wl)
    s_nan = s.copy()
    for k in range(s.shape[0]):
        flagged = np.abs(s[k]).sum(0) == 0
        assert flagged.any()
        s_nan[k][:, flagged] = np.nan
        s_nan[k][flagged, :] = np.nan
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis, tolerance=1e-6)
    pl.process(s, xyz, wl)
    a = pl.images()
    pl.reset()
    pl.process(s_nan, xyz, wl)
    b = pl.images()
    assert np.all(np.isfinite(b))
    assert _rel_l2(b, a.astype(np.float64)) <= 1e-6
    bad = s.copy()
    kept = np.nonzero(np.abs(s[1]).sum(0) > 0)[0]
    bad[1][kept[-1], kept[0]] = bad[1][kept[0], kept[-1]] = np.nan
    with pytest.raises(bipp.EigensolverError):
        pl.process(bad, xyz, wl)
    assert np.array_equal(pl.images(), b)
    pl.close()


@pytest.mark.parametrize("filt", ["std", "sqrt", "inv", "inv_sqrt"])
def test_pipeline_filters_vs_fp64_oracle(ctx, filt):
    """The reference's eigenvalue filters (python/bipp/filter.py:7-51: level mask, then the
    filter) through the batched pipeline, on two positive levels and one negative level
    whose bounds sit in wide gaps of the spectra; a wrong filter is off by O(1)."""
    import bipp_b200 as bipp

    cfg, obs, s, xyz = _pipeline_case(n_ant=32, n_steps=3, image=24)
    dmax = bb.eigh_gram(cfg.wl, s[0], np.eye(cfg.n_antenna), xyz[0])[1].max()
    intervals = np.array([[0.2, np.inf], [0.02, 0.2], [-0.11, -0.02]]) * dmax
    intervals[0, 1] = np.inf
    ref_img, steps = _oracle_pipeline(cfg, obs, s, xyz, intervals, filt)
    for st in steps:
        for lo, hi in intervals:
            assert ((st["d"] >= lo) & (st["d"] <= hi)).sum() >= 2
    n = cfg.image_size
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, _lattice(obs, n), obs.lmn[:, 2], obs.basis, tolerance=1e-6,
                       filter=filt)
    pl.process(s, xyz, np.full(s.shape[0], cfg.wl))
    img = pl.images()
    pl.close()
    for lv in range(intervals.shape[0]):
        assert _rel_l2(img[lv], ref_img[:, lv]) <= 1e-3, (lv, _rel_l2(img[lv], ref_img[:, lv]))
