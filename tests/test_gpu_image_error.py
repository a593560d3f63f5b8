"""Image error of the batched pipeline against the FP64 oracle, at three workload shapes.

- benchmark shape: 512 antennas (380-512 kept per step), 200 sources, 4 energy levels,
  1024 x 1024 pixels over 16 degrees, NUFFT tolerance 1e-5; four time steps spread over
  the 4.5-hour observation (so that the w extent is the full one).
- precision study: 550 antennas to 65 km, wavelength 0.21 m, 1000 sources, 8 levels,
  4096 x 4096 pixels over 4 degrees, NUFFT tolerance 1e-6; one time step, 16,384 pixels.
- full pipeline: 1024 antennas to 50 km with 25% flagged, 8 frequency channels
  (1.5-3 m), 500 sources, 8 levels, 2048 x 2048 pixels over 16 degrees, tolerance 1e-5;
  two time steps x two channels (the extreme wavelengths) in one batch.

FP32 visibilities go through the pipeline; the oracle is the compiled reference (FP64
zhegv eigensolver, virtual_vis, and the exact direct sum nuft_sum in FP64) on random
pixels. Tolerance: 1e-4 relative L2 over the level stack (the metric's image-error bar).
"""
import numpy as np
import pytest

from oracle import bluebild as bb
from oracle import ref

pytestmark = pytest.mark.gpu


def _image_error(ctx, cfg, entries, n_pix, chunk):
    """entries: (time step, channel) pairs, all imaged in one pipeline batch."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    wls = cfg.wavelengths()
    s_l, x_l, w_l = [], [], []
    for step, ch in entries:
        s, x = sim.visibilities(obs, [step], masks=masks, wl=float(wls[ch]), noise_key=ch)
        s_l.append(s.numpy()[0])
        x_l.append(x.numpy()[0])
        w_l.append(float(wls[ch]))
    s, xyz, wl = np.stack(s_l), np.stack(x_l), np.array(w_l)
    N = cfg.n_antenna
    # FP64 reference eigenpairs of every entry
    eig = []
    for k in range(len(entries)):
        v, d, nr, sc = ref.eigh_gram(wl[k], s[k].astype(np.complex128), np.eye(N), xyz[k], dtype=np.float64)
        eig.append((v, d, sc))
    intervals = bb.infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, np.concatenate([e[1] for e in eig]))
    n = cfg.image_size
    lmn = obs.lmn
    l = lmn[:, 0].reshape(n, n)
    m = lmn[:, 1].reshape(n, n)
    lattice = (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])
    pl = bipp.Pipeline(ctx, N, intervals, lattice, lmn[:, 2], obs.basis, tolerance=cfg.eps, chunk_steps=chunk)
    pl.process(s, xyz, wl)
    img = pl.images()
    pl.close()
    # oracle on a pixel subset
    pix = np.random.default_rng(33).choice(lmn.shape[0], n_pix, replace=False)
    x, y, z = lmn[pix, 0], lmn[pix, 1], lmn[pix, 2]
    out = np.zeros((intervals.shape[0], n_pix))
    for k, (v, d, sc) in enumerate(eig):
        au = xyz[k] @ obs.basis
        b = (au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3) * (bb.TWO_PI / wl[k])
        for lv in range(intervals.shape[0]):
            dl = bb.level_eigenvalues(d, intervals[lv, 0], intervals[lv, 1])
            vv = bb.virtual_vis(sc, dl, v).reshape(-1, order="F")
            ref.nuft_sum(1.0, vv, b[:, 0], b[:, 1], b[:, 2], x, y, z, out=out[lv])
    out /= len(entries)
    got = img[:, pix].astype(np.float64)
    return np.linalg.norm(got - out) / np.linalg.norm(out)


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_at_benchmark_shape(ctx):
    from bipp_b200 import simulate as sim

    err = _image_error(ctx, sim.config_c2(), [(0, 0), (683, 0), (1366, 0), (2047, 0)], 2048, 4)
    assert err <= 1e-4, err


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_precision_study(ctx):
    from bipp_b200 import simulate as sim

    err = _image_error(ctx, sim.config_c3(), [(0, 0)], 16384, 1)
    assert err <= 1e-4, err


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_multichannel_1024_antennas(ctx):
    from bipp_b200 import simulate as sim

    cfg = sim.config_c5()
    err = _image_error(ctx, cfg, [(0, 0), (0, 7), (4095, 0), (4095, 7)], 512, 4)
    assert err <= 1e-4, err
