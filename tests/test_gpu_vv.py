"""GPU: the virtual-visibility products VV_l = X diag(filter(d) / nVis) X^H of the batched
pipeline (src/host/virtual_vis.cpp:52-68) in its four arithmetic modes: 3xTF32 and BF16x3
on the tensor cores (tcgen05), FP32 and FP64 on the CUDA cores.

The level images of one batch (512 antennas with flagging, 4 levels, one of them empty)
agree between the modes: 3xTF32 and FP32 with FP64 to 1e-5 relative L2 per level, BF16x3
to 1e-4; a level whose interval holds no eigenvalue gives an image that is exactly zero
(the reference's VV = 0, src/host/virtual_vis.cpp:35-43)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_vv_precision_modes_agree(ctx):
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim
    from bipp_b200.parameter_estimator import infer_intervals

    cfg = sim.config_c2(n_steps=2048)
    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    steps = [0, 300, 700, 1100, 1500, 2047]
    s, xyz = sim.visibilities(obs, steps, masks=masks)
    s, xyz = s.numpy(), xyz.numpy()
    wl = np.full(len(steps), cfg.wl)
    _, d, _, _ = bipp.eigh_gram_batched(wl.astype(np.float32), s, xyz, ctx=ctx)
    iv = infer_intervals(3, 1.0, "log", 0.0, np.inf, d)
    intervals = np.vstack([iv, [[1e12, 1e13]]])   # the last level holds no eigenvalue
    n = 256
    lmn = obs.lmn
    grid = cfg.image_size
    l = lmn[:, 0].reshape(grid, grid)
    m = lmn[:, 1].reshape(grid, grid)
    # a coarser lattice over the same field keeps the NUFFT small
    step = grid // n
    lat = (n, n, l[0, 0], m[0, 0], step * (l[1, 0] - l[0, 0]), step * (l[0, 1] - l[0, 0]),
           step * (m[1, 0] - m[0, 0]), step * (m[0, 1] - m[0, 0]))
    pn = lmn[:, 2].reshape(grid, grid)[::step, ::step].reshape(-1)
    imgs = {}
    for mode in ("fp64", "tf32x3", "bf16x3", "fp32"):
        pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, lat, pn, obs.basis, tolerance=1e-6, chunk_steps=4,
                           vv_precision=mode)
        pl.process(s, xyz, wl)
        imgs[mode] = pl.images().astype(np.float64)
        pl.close()
    ref = imgs["fp64"]
    assert np.all(ref[3] == 0)
    for mode, tol in (("tf32x3", 1e-5), ("fp32", 1e-5), ("bf16x3", 1e-4)):
        assert np.all(imgs[mode][3] == 0), mode
        for lv in range(3):
            err = np.linalg.norm(imgs[mode][lv] - ref[lv]) / np.linalg.norm(ref[lv])
            print(f"{mode} level {lv}: {err:.2e}")
            assert err <= tol, (mode, lv, err)
