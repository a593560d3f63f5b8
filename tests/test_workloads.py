"""Host-side logic of the benchmark workloads (no GPU): the bytes a host-input pipeline
call copies, the seeded workload configurations and the per-workload bench defaults."""
import sys

import numpy as np

import bench
from bipp_b200 import simulate as sim


def test_lower_block_bytes_counts_the_copied_elements():
    # the library copies, per 64-column block, rows from the block's diagonal row down
    for n, t in [(512, 1), (300, 3), (64, 2), (65, 1), (1024, 2)]:
        mask = np.zeros((n, n), dtype=bool)   # [row, column]
        for c0 in range(0, n, 64):
            mask[c0:, c0:c0 + 64] = True
        assert bench.lower_block_bytes(n, t) == t * 8 * int(mask.sum())
        # the whole lower triangle is covered
        assert mask[np.tril_indices(n)].all()
    assert bench.lower_block_bytes(512, 1) == 0.5625 * 512 * 512 * 8


def test_workload_configs():
    c2 = sim.config_c2()
    assert (c2.n_antenna, c2.n_steps, c2.image_size, c2.n_levels, c2.eps) == (512, 2048, 1024, 4, 1e-5)
    assert c2.keep == (380, 512) and c2.n_channels == 1
    c3 = sim.config_c3()
    assert (c3.n_antenna, c3.wl, c3.n_src, c3.n_levels, c3.image_size, c3.eps) == (550, 0.21, 1000, 8, 4096, 1e-6)
    c5 = sim.config_c5()
    assert (c5.n_antenna, c5.n_steps, c5.n_channels, c5.n_src, c5.n_levels, c5.image_size) == (1024, 4096, 8, 500, 8,
                                                                                                 2048)
    assert c5.keep == (768, 768)   # 25 % flagged per step
    wl = c5.wavelengths()
    assert wl.shape == (8,) and wl[0] == 1.5 and wl[-1] == 3.0 and np.all(np.diff(wl) > 0)
    assert np.all(c2.wavelengths() == 2.0)


def test_channel_noise_differs_per_channel():
    cfg = sim.config_c5(n_antenna=24, n_steps=2, keep=None, image_size=16)
    obs = sim.observation(cfg)
    a, _ = sim.visibilities(obs, [0], wl=2.0, noise_key=0)
    b, _ = sim.visibilities(obs, [0], wl=2.0, noise_key=1)
    c, _ = sim.visibilities(obs, [0], wl=2.0, noise_key=0)
    assert np.array_equal(a.numpy(), c.numpy())      # seeded
    assert not np.array_equal(a.numpy(), b.numpy())  # channels draw their own noise


def test_bench_defaults_per_workload(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    a = bench.parse()
    assert (a.workload, a.time_steps, a.antennas, a.image, a.chunk_steps) == ("c2", 2048, 512, 1024, 2048)
    monkeypatch.setattr(sys, "argv", ["bench.py", "--workload", "c5"])
    a = bench.parse()
    assert (a.time_steps, a.antennas, a.image, a.chunk_steps) == (128, 1024, 2048, 592)
    assert bench.metric_of(a) == bench.METRIC_C5


def test_geometry_matches_reference_frame():
    """The workload generator's UVW frame, pixel grid and baseline order against the
    reference's own python/bipp/frame.py (uvw_basis, make_grids, reshape_uvw) run on the
    same inputs (tests/golden/frame.npz)."""
    import types

    from conftest import golden

    g = golden("frame.npz")
    for k, (lon, lat) in enumerate(g["centres"]):
        assert np.allclose(sim.uvw_basis(lon, lat), g[f"basis_{k}"], rtol=0, atol=1e-15)
    for k, (n, fov) in enumerate(g["grids"]):
        assert np.allclose(sim.make_lmn_grid(int(n), fov), g[f"lmn_{k}"].T, rtol=0, atol=1e-15)
    # baseline k = i + j N <-> U_i - U_j, as reshape_uvw orders it (float32 output)
    obs = types.SimpleNamespace(basis=np.eye(3))
    got = sim.baseline_uvw(obs, g["antenna_uvw"])
    assert got.dtype == np.float32
    assert np.allclose(got, g["uvw_reshaped"], rtol=1e-6, atol=1e-4)
