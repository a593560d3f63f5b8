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

At the benchmark's batch size (256 of the 2048 steps, so that the NUFFT splits heavy
tiles and the w axis into several slabs) the FP64 reference is the library's own FP64
pieces (bipp_b200.verify), which are first checked against the compiled reference.
"""
import numpy as np
import pytest

from oracle import bluebild as bb
from oracle import ref

pytestmark = pytest.mark.gpu


def _image_error(ctx, cfg, entries, n_pix, chunk, modes=None):
    """entries: (time step, channel) pairs, all imaged in one pipeline batch. With
    `modes` (virtual-visibility precisions) the error of each mode is returned as a dict,
    the oracle computed once."""
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
    imgs = {}
    for mode in (modes or ("tf32x3",)):
        pl = bipp.Pipeline(ctx, N, intervals, lattice, lmn[:, 2], obs.basis, tolerance=cfg.eps, chunk_steps=chunk,
                           vv_precision=mode)
        pl.process(s, xyz, wl)
        imgs[mode] = pl.images()
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
    errs = {m: np.linalg.norm(img[:, pix].astype(np.float64) - out) / np.linalg.norm(out) for m, img in imgs.items()}
    return errs if modes else errs["tf32x3"]


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_at_benchmark_shape(ctx):
    from bipp_b200 import simulate as sim

    err = _image_error(ctx, sim.config_c2(), [(0, 0), (683, 0), (1366, 0), (2047, 0)], 2048, 4)
    assert err <= 1e-4, err


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_precision_study(ctx):
    """The precision study (550 antennas, 8 levels, 4096^2 px, tolerance 1e-6, 16,384
    random pixels, seed 33): the virtual-visibility products in FP64, 3xTF32 and BF16x3 on
    the tensor cores, and FP32 on the CUDA cores; every mode's image within 1e-4 relative
    L2 of the FP64 oracle, and the split tensor-core modes within 2x of the FP64 mode's
    error (what the rest of the FP32 pipeline leaves) plus 1e-5."""
    from bipp_b200 import simulate as sim

    errs = _image_error(ctx, sim.config_c3(), [(0, 0)], 16384, 1, modes=("fp64", "tf32x3", "bf16x3", "fp32"))
    print("precision study image errors:", {m: f"{e:.3e}" for m, e in errs.items()})
    for m, e in errs.items():
        assert e <= 1e-4, (m, errs)
    for m in ("tf32x3", "bf16x3"):
        assert errs[m] <= 2 * errs["fp64"] + 1e-5, errs


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_multichannel_1024_antennas(ctx):
    from bipp_b200 import simulate as sim

    cfg = sim.config_c5()
    err = _image_error(ctx, cfg, [(0, 0), (0, 7), (4095, 0), (4095, 7)], 512, 4)
    assert err <= 1e-4, err


def _c2_steps_on_device(cfg, steps):
    """S (each step's matrix in column-major order), xyz, wl of the given steps on cuda:0."""
    import torch

    from bipp_b200 import simulate as sim

    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    dev = torch.device("cuda", 0)
    N = cfg.n_antenna
    S = torch.empty((len(steps), N, N), dtype=torch.complex64, device=dev)
    xyz = torch.empty((len(steps), N, 3), dtype=torch.float64, device=dev)
    for i0 in range(0, len(steps), 64):
        part = steps[i0:i0 + 64]
        s, x = sim.visibilities(obs, part, device=dev, dtype=torch.complex64, masks=masks, wl=cfg.wl)
        S[i0:i0 + len(part)] = s.transpose(1, 2)
        xyz[i0:i0 + len(part)] = x
    wl = torch.full((len(steps),), float(cfg.wl), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    return obs, S, xyz, wl


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_fp64_check_pieces_against_compiled_reference(ctx):
    """The FP64 image check of bipp_b200.verify (FP64 batched eigensolve, FP64 virtual
    visibilities, direct sum with FP64 trigonometry) equals the compiled reference's
    zhegv + virtual_vis + nuft_sum<double> on two steps of the benchmark's workload (512
    antennas, 4 levels): eigenvalues to 1e-10, level images to 1e-6 relative L2 (the check
    rounds VV to complex64, a 6e-8 relative perturbation)."""
    from bipp_b200 import simulate as sim
    from bipp_b200 import verify

    cfg = sim.config_c2()
    obs, S, xyz, wl = _c2_steps_on_device(cfg, [5, 1500])
    s_log = S.transpose(1, 2).cpu().numpy().astype(np.complex128)
    x, w = xyz.cpu().numpy(), wl.cpu().numpy()
    eig = [ref.eigh_gram(w[k], s_log[k], np.eye(cfg.n_antenna), x[k], dtype=np.float64) for k in range(2)]
    intervals = bb.infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, np.concatenate([e[1] for e in eig]))
    pix = np.random.default_rng(3).choice(obs.lmn.shape[0], 64, replace=False)
    got, d64 = verify.fp64_level_images(ctx, s_log, x, w, obs.basis, intervals, obs.lmn[pix])
    out = np.zeros((cfg.n_levels, 64))
    for k, (v, d, nr, sc) in enumerate(eig):
        assert np.abs(d64[k] - d).max() <= 1e-10 * np.abs(d).max()
        au = x[k] @ obs.basis
        b = (au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3) * (bb.TWO_PI / w[k])
        for lv in range(cfg.n_levels):
            vv = bb.virtual_vis(sc, bb.level_eigenvalues(d, intervals[lv, 0], intervals[lv, 1]), v).reshape(-1, order="F")
            ref.nuft_sum(1.0, vv, b[:, 0], b[:, 1], b[:, 2], obs.lmn[pix, 0], obs.lmn[pix, 1], obs.lmn[pix, 2],
                         out=out[lv])
    out /= 2
    assert np.linalg.norm(got - out) / np.linalg.norm(out) <= 1e-6


def test_pipeline_image_error_benchmark_batch(ctx):
    """256 of the benchmark's 2048 time steps (every 8th, so the w extent is the full one)
    imaged as one batch, as the benchmark does: the NUFFT splits heavy tiles into parts
    that accumulate with atomics and processes the w axis in several slabs (both asserted
    from the pipeline's statistics); image error at 512 random pixels <= 1e-4 relative
    L2 against the FP64 check; the eigenvalues inside the level range within 1e-5 of FP64
    normwise and, for those above 1e-2 of their step's largest, per eigenvalue (relative;
    the smaller ones carry the FP32 solver's absolute error, as the reference's own FP32
    path does, and are covered by the normwise bound)."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim
    from bipp_b200 import verify
    from bipp_b200.parameter_estimator import infer_intervals

    cfg = sim.config_c2()
    obs, S, xyz, wl = _c2_steps_on_device(cfg, list(range(0, cfg.n_steps, 8)))
    _, d, _, _ = bipp.eigh_gram_batched(wl[:32].cpu().numpy().astype(np.float32),
                                        S[:32].transpose(1, 2).cpu().numpy(), xyz[:32].cpu().numpy(), ctx=ctx)
    intervals = infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, d)
    r = verify.check_batch(ctx, S, xyz, wl, obs, cfg.image_size, intervals, cfg.eps, n_pix=512)
    print(r)
    assert r["split_tiles"] > 0 and r["slabs"] > 1, r
    assert r["image_rel_l2"] <= 1e-4, r
    assert r["eig_rel_err_normwise"] <= 1e-5, r
    assert r["eig_rel_err_max_above_1e-2"] <= 1e-5, r
