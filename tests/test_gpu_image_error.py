"""Image error of the batched pipeline at the benchmark's shape against the FP64 oracle.

The benchmark workload: 512 antennas (380-512 kept per step), 200 sources, 4 energy
levels, 1024 x 1024 pixels over 16 degrees, NUFFT tolerance 1e-5, FP32 visibilities.
Four time steps spread over the 4.5-hour observation (so that the w extent is the full
one) go through the pipeline; the oracle is the compiled reference (FP64 zhegv
eigensolver, virtual_vis, and the exact direct sum nuft_sum in FP64) on 2048 random
pixels. Tolerance: 1e-4 relative L2 over the level stack (the metric's image-error bar).
"""
import numpy as np
import pytest

from oracle import bluebild as bb
from oracle import ref

pytestmark = pytest.mark.gpu

STEPS = [0, 683, 1366, 2047]
N_PIX = 2048


@pytest.mark.skipif(not ref.available(), reason="compiled reference oracle not built")
def test_pipeline_image_error_at_benchmark_shape(ctx):
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    cfg = sim.config_c2()
    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    s, xyz = sim.visibilities(obs, STEPS, masks=masks)
    s, xyz = s.numpy(), xyz.numpy()
    N = cfg.n_antenna
    # FP64 reference eigenpairs of every step
    eig = []
    for k in range(len(STEPS)):
        v, d, nr, sc = ref.eigh_gram(cfg.wl, s[k].astype(np.complex128), np.eye(N), xyz[k], dtype=np.float64)
        eig.append((v, d, sc))
    intervals = bb.infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, np.concatenate([e[1] for e in eig]))
    # pipeline over the full 1024^2 image
    n = cfg.image_size
    lmn = obs.lmn
    l = lmn[:, 0].reshape(n, n)
    m = lmn[:, 1].reshape(n, n)
    lattice = (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])
    pl = bipp.Pipeline(ctx, N, intervals, lattice, lmn[:, 2], obs.basis, tolerance=cfg.eps, chunk_steps=4)
    pl.process(s, xyz, np.full(len(STEPS), cfg.wl))
    img = pl.images()
    pl.close()
    # oracle on a pixel subset
    pix = np.random.default_rng(33).choice(lmn.shape[0], N_PIX, replace=False)
    x, y, z = lmn[pix, 0], lmn[pix, 1], lmn[pix, 2]
    out = np.zeros((intervals.shape[0], N_PIX))
    for k, (v, d, sc) in enumerate(eig):
        au = xyz[k] @ obs.basis
        b = (au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3) * (bb.TWO_PI / cfg.wl)
        for lv in range(intervals.shape[0]):
            dl = bb.level_eigenvalues(d, intervals[lv, 0], intervals[lv, 1])
            vv = bb.virtual_vis(sc, dl, v).reshape(-1, order="F")
            ref.nuft_sum(1.0, vv, b[:, 0], b[:, 1], b[:, 2], x, y, z, out=out[lv])
    out /= len(STEPS)
    got = img[:, pix].astype(np.float64)
    err = np.linalg.norm(got - out) / np.linalg.norm(out)
    assert err <= 1e-4, err
