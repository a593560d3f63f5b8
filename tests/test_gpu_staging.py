"""GPU: the double-buffered host input of the batched pipeline (bipp_pipeline_stage /
bipp_pipeline_process_staged): two batches staged ahead from pinned host memory give the
same level images as the synchronous host-input call (1e-6 relative L2; only the
summation order of atomics may differ), a third stage with two batches waiting is
refused, and processing with nothing staged is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_staged_batches_match_host_calls(ctx):
    import torch

    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim
    from bipp_b200.parameter_estimator import infer_intervals

    cfg = sim.config_c2(n_antenna=128, n_steps=48, image_size=128, n_src=60, keep=(100, 128))
    obs = sim.observation(cfg)
    s, x = sim.visibilities(obs, list(range(48)), masks=sim.keep_masks(cfg))
    S = np.ascontiguousarray(np.transpose(s.numpy().astype(np.complex64), (0, 2, 1)))
    Sp = torch.from_numpy(S).pin_memory()
    Xp = torch.from_numpy(np.ascontiguousarray(x.numpy(), dtype=np.float64)).pin_memory()
    Wp = torch.full((48,), cfg.wl, dtype=torch.float64).pin_memory()
    _, d, _, _ = bipp.eigh_gram_batched(np.full(8, cfg.wl, np.float32), s[:8].numpy(), x[:8].numpy(), ctx=ctx)
    intervals = infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, d)
    n = cfg.image_size
    l = obs.lmn[:, 0].reshape(n, n)
    m = obs.lmn[:, 1].reshape(n, n)
    lat = (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, lat, obs.lmn[:, 2], obs.basis, tolerance=cfg.eps,
                       chunk_steps=24, max_steps=24)
    es = Sp[0].numel() * 8
    ex, ew = Xp[0].numel() * 8, 8
    halves = [(Sp.data_ptr() + h * 24 * es, Xp.data_ptr() + h * 24 * ex, Wp.data_ptr() + h * 24 * ew) for h in (0, 1)]
    ref = []
    for sp, xp, wp in halves:
        pl.reset()
        pl.process_host_ptr(24, sp, xp, wp)
        ref.append(pl.images().astype(np.float64))
    with pytest.raises(bipp.BippError):
        pl.process_staged()
    pl.stage_host_ptr(24, *halves[0])
    pl.stage_host_ptr(24, *halves[1])
    with pytest.raises(bipp.InvalidParameterError):
        pl.stage_host_ptr(24, *halves[0])
    for h in (0, 1):
        pl.reset()
        pl.process_staged()
        got = pl.images().astype(np.float64)
        for lv in range(got.shape[0]):
            assert np.linalg.norm(got[lv] - ref[h][lv]) <= 1e-6 * np.linalg.norm(ref[h][lv]), (h, lv)
    pl.close()
