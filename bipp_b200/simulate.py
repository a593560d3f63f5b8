"""Seeded synthetic Bluebild inputs (antenna layouts, skies, visibilities, uvw, pixel grids).

The formulas restate the semantics of the reference's simulation helpers, which
need astropy and network catalogues that are absent here:

* visibilities  S_ij = sum_q I_q exp(-i 2 pi/wl r_q . (p_i - p_j)) + noise, with the
  diagonal (autocorrelations) zeroed - python/bipp/statistics.py:55, 110-120;
* UVW frame basis and the l-fastest pixel grid - python/bipp/frame.py:9-72;
* baseline ordering k = i + j nAnt <-> uvw = p_i - p_j in the UVW frame -
  python/bipp/frame.py:75-89, python/bipp/instrument.py:246-247;
* Gram matrix G = sinc(2|p_i - p_j|/wl) - src/host/gram_matrix.cpp:23-56.

Geometry choices not fixed by the workload descriptions: array latitude -30 deg,
phase centre at the zenith at mid-observation (RA 0, dec = latitude), Earth
rotation 7.2921e-5 rad/s about the celestial pole, "X km disc" = diameter X,
"log-radial to R" = radius log-uniform in [10 m, R] with uniform azimuth.
Flagged antennas are zero rows/columns of S (src/eigensolver.cpp:148-175).

torch is used only as an array library here (CPU or GPU) so that the large
workloads can be generated quickly; nothing in this module is on the timed path.
"""
from __future__ import annotations

import dataclasses
import math
from typing import Optional, Sequence, Tuple

import numpy as np
import torch

EARTH_OMEGA = 7.2921e-5  # rad/s


@dataclasses.dataclass
class SimConfig:
    name: str
    n_antenna: int
    layout: str                 # "disc" | "logradial"
    extent_m: float             # disc diameter or log-radial max radius
    z_spread_m: float
    wl: float
    n_steps: int
    dt_s: float
    n_src: int
    flux: Tuple[float, float]
    src_radius_deg: float
    noise_sigma: float
    n_levels: int
    image_size: int
    fov_deg: float
    eps: float
    keep: Optional[Tuple[int, int]] = None   # per-step kept-antenna count range (inclusive)
    latitude_deg: float = -30.0
    seed: int = 0
    double: bool = False
    n_channels: int = 1                      # frequency channels per time step
    wl_range: Optional[Tuple[float, float]] = None   # channel wavelengths, linearly spaced

    def wavelengths(self) -> np.ndarray:
        """(n_channels,) wavelengths in metres."""
        if self.n_channels == 1 or self.wl_range is None:
            return np.full(self.n_channels, self.wl)
        return np.linspace(self.wl_range[0], self.wl_range[1], self.n_channels)


def config_c1(**kw) -> SimConfig:
    """Plain Bluebild, CPU-runnable, complex128: 60 antennas in a 3 km disc."""
    c = SimConfig(name="c1_n60_256px", n_antenna=60, layout="disc", extent_m=3000.0,
                  z_spread_m=10.0, wl=2.0, n_steps=16, dt_s=8.0, n_src=20, flux=(0.1, 10.0),
                  src_radius_deg=5.0, noise_sigma=0.01, n_levels=2, image_size=256,
                  fov_deg=10.0, eps=1e-7, keep=None, seed=1, double=True)
    return dataclasses.replace(c, **kw)


def config_c2(**kw) -> SimConfig:
    """Batched uneven steps: 512 antennas log-radial to 35 km, 2048 steps with
    380-512 antennas kept per step, 200 sources within 8 deg, 4 levels, 1024^2 px."""
    c = SimConfig(name="c2_n512_1024px", n_antenna=512, layout="logradial", extent_m=35000.0,
                  z_spread_m=10.0, wl=2.0, n_steps=2048, dt_s=8.0, n_src=200, flux=(0.01, 10.0),
                  src_radius_deg=8.0, noise_sigma=0.01, n_levels=4, image_size=1024,
                  fov_deg=16.0, eps=1e-5, keep=(380, 512), seed=2, double=False)
    return dataclasses.replace(c, **kw)


def config_c3(**kw) -> SimConfig:
    """Precision study on one large step: 550 antennas log-radial to 65 km, wl 0.21 m,
    1000 sources (0.001-1 Jy), 8 levels, 4096^2 px, NUFFT eps 1e-6."""
    c = SimConfig(name="c3_n550_4096px", n_antenna=550, layout="logradial", extent_m=65000.0,
                  z_spread_m=10.0, wl=0.21, n_steps=1, dt_s=8.0, n_src=1000, flux=(0.001, 1.0),
                  src_radius_deg=2.0, noise_sigma=0.01, n_levels=8, image_size=4096,
                  fov_deg=4.0, eps=1e-6, keep=None, seed=3, double=False)
    return dataclasses.replace(c, **kw)


def config_c5(**kw) -> SimConfig:
    """Full pipeline: 1024 antennas log-radial to 50 km, 25% flagged per step, 4096 steps
    x 8 channels (wl 1.5-3 m), 500 sources (0.001-10 Jy), 8 levels, 2048^2 px, eps 1e-5."""
    c = SimConfig(name="c5_n1024_2048px", n_antenna=1024, layout="logradial", extent_m=50000.0,
                  z_spread_m=10.0, wl=2.0, n_steps=4096, dt_s=8.0, n_src=500, flux=(0.001, 10.0),
                  src_radius_deg=8.0, noise_sigma=0.01, n_levels=8, image_size=2048,
                  fov_deg=16.0, eps=1e-5, keep=(768, 768), seed=5, double=False, n_channels=8,
                  wl_range=(1.5, 3.0))
    return dataclasses.replace(c, **kw)


def config_c4(**kw) -> SimConfig:
    """Learned rank predictor: 256 antennas in a 10 km disc, 10,000 time steps, each with
    its own sky of 5-200 sources (0.01-10 Jy) within 8 deg and its own noise level,
    log-uniform in 0.001-0.1 (c4_step_sky); n_src is the largest source count."""
    c = SimConfig(name="c4_n256_rank", n_antenna=256, layout="disc", extent_m=10000.0,
                  z_spread_m=10.0, wl=2.0, n_steps=10000, dt_s=8.0, n_src=200, flux=(0.01, 10.0),
                  src_radius_deg=8.0, noise_sigma=0.01, n_levels=4, image_size=256,
                  fov_deg=16.0, eps=1e-5, keep=None, seed=4, double=False)
    return dataclasses.replace(c, **kw)


C4_SOURCES = (5, 200)
C4_SIGMA = (0.001, 0.1)


def c4_step_sky(obs: "Observation", step: int):
    """Sky and noise level of one step of the rank-predictor workload: Q ~ U{5..200}
    sources uniform on the cap of radius src_radius_deg, log-uniform fluxes, and sigma
    log-uniform in [0.001, 0.1]. Returns (directions (Q, 3), fluxes (Q,), sigma)."""
    cfg = obs.cfg
    rng = np.random.default_rng([cfg.seed, 4000, int(step)])
    q = int(rng.integers(C4_SOURCES[0], C4_SOURCES[1] + 1))
    cos_rho = math.cos(math.radians(cfg.src_radius_deg))
    ca = rng.uniform(cos_rho, 1.0, q)
    sa = np.sqrt(1 - ca ** 2)
    az = rng.uniform(0, 2 * np.pi, q)
    dirs = np.stack([sa * np.cos(az), sa * np.sin(az), ca], axis=1) @ obs.basis.T
    flux = np.exp(rng.uniform(np.log(cfg.flux[0]), np.log(cfg.flux[1]), q))
    sigma = float(np.exp(rng.uniform(np.log(C4_SIGMA[0]), np.log(C4_SIGMA[1]))))
    return dirs, flux, sigma


def visibilities_c4(obs: "Observation", steps: Sequence[int], device="cpu",
                    dtype=torch.complex64) -> Tuple[torch.Tensor, torch.Tensor]:
    """S (len(steps), N, N) and positions (len(steps), N, 3) of rank-predictor steps, each
    with its own sky and noise level (c4_step_sky); otherwise as visibilities()."""
    cfg = obs.cfg
    n, B, qmax = cfg.n_antenna, len(steps), C4_SOURCES[1]
    dirs = np.zeros((B, qmax, 3))
    flux = np.zeros((B, qmax))
    sig = np.zeros(B)
    for i, st in enumerate(steps):
        d, f, sg = c4_step_sky(obs, st)
        dirs[i, :len(f)] = d
        flux[i, :len(f)] = f
        sig[i] = sg
    xyz = np.stack([obs.positions(s) for s in steps])
    xyz_t = torch.from_numpy(xyz).to(device)
    ph = (2 * math.pi / cfg.wl) * torch.einsum("bqc,bnc->bqn", torch.from_numpy(dirs).to(device), xyz_t)
    a = torch.polar(torch.ones_like(ph), ph)
    fl = torch.from_numpy(flux).to(device).to(a.dtype)
    s = torch.einsum("bqi,bq,bqj->bij", a.conj(), fl, a)
    g = torch.Generator(device=device)
    g.manual_seed(cfg.seed * 1000003 + int(steps[0]) + 104729)
    sg = torch.from_numpy(sig / math.sqrt(2.0)).to(device)[:, None, None]
    xr = torch.randn((B, n, n), generator=g, device=device, dtype=torch.float64) * sg
    xi = torch.randn((B, n, n), generator=g, device=device, dtype=torch.float64) * sg
    x = torch.complex(xr, xi)
    s = s + 0.5 * (x + x.conj().transpose(1, 2))
    s.diagonal(dim1=1, dim2=2).zero_()
    return s.to(dtype), xyz_t


# --- geometry -----------------------------------------------------------------------

def antenna_layout_enu(cfg: SimConfig) -> np.ndarray:
    """(N, 3) east/north/up positions in metres."""
    rng = np.random.default_rng(cfg.seed)
    n = cfg.n_antenna
    az = rng.uniform(0.0, 2 * np.pi, n)
    if cfg.layout == "disc":
        r = (cfg.extent_m / 2.0) * np.sqrt(rng.uniform(0.0, 1.0, n))
    elif cfg.layout == "logradial":
        r = np.exp(rng.uniform(np.log(10.0), np.log(cfg.extent_m), n))
    else:
        raise ValueError(cfg.layout)
    z = rng.uniform(-cfg.z_spread_m, cfg.z_spread_m, n)
    return np.stack([r * np.cos(az), r * np.sin(az), z], axis=1)


def enu_to_celestial(enu: np.ndarray, lat_rad: float, theta: float) -> np.ndarray:
    """Positions in the inertial (celestial) frame at sidereal angle theta."""
    st, ct = math.sin(theta), math.cos(theta)
    sp, cp = math.sin(lat_rad), math.cos(lat_rad)
    e = np.array([-st, ct, 0.0])
    nn = np.array([-sp * ct, -sp * st, cp])
    u = np.array([cp * ct, cp * st, sp])
    return enu[:, 0:1] * e + enu[:, 1:2] * nn + enu[:, 2:3] * u


def uvw_basis(lon_rad: float, lat_rad: float) -> np.ndarray:
    """(3, 3) matrix whose columns are the U, V, W directions
    (python/bipp/frame.py:9-37)."""
    w_dir = np.array([math.cos(lat_rad) * math.cos(lon_rad), math.cos(lat_rad) * math.sin(lon_rad),
                      math.sin(lat_rad)])
    u_dir = np.array([-math.sin(lon_rad), math.cos(lon_rad), 0.0])
    v_dir = np.array([-math.cos(lon_rad) * math.sin(lat_rad), -math.sin(lon_rad) * math.sin(lat_rad),
                      math.cos(lat_rad)])
    return np.stack([u_dir, v_dir, w_dir], axis=-1)


def make_lmn_grid(grid_size: int, fov_rad: float) -> np.ndarray:
    """(P, 3) pixel lmn with l fastest, half-pixel offset grid of
    python/bipp/frame.py:55-72."""
    lim = math.sin(fov_rad / 2)
    offset = lim / (grid_size / 2) * 0.5
    s1 = np.linspace(-lim - offset, lim - offset, grid_size)
    s2 = np.linspace(-lim + offset, lim + offset, grid_size)
    l_grid, m_grid = np.meshgrid(s2, s1)
    n_grid = np.sqrt(1 - l_grid ** 2 - m_grid ** 2)
    return np.stack([l_grid.reshape(-1), m_grid.reshape(-1), n_grid.reshape(-1)], axis=1)


def sky(cfg: SimConfig, basis: np.ndarray):
    """Source directions (celestial frame, unit vectors) uniform on the spherical
    cap of radius src_radius_deg about the phase centre; log-uniform fluxes."""
    rng = np.random.default_rng(cfg.seed + 1000)
    n = cfg.n_src
    cos_rho = math.cos(math.radians(cfg.src_radius_deg))
    ca = rng.uniform(cos_rho, 1.0, n)
    sa = np.sqrt(1 - ca ** 2)
    az = rng.uniform(0, 2 * np.pi, n)
    lmn = np.stack([sa * np.cos(az), sa * np.sin(az), ca], axis=1)
    dirs = lmn @ basis.T
    flux = np.exp(rng.uniform(np.log(cfg.flux[0]), np.log(cfg.flux[1]), n))
    return dirs, flux


@dataclasses.dataclass
class Observation:
    cfg: SimConfig
    basis: np.ndarray          # (3,3) UVW basis (columns)
    enu: np.ndarray            # (N,3)
    src_dirs: np.ndarray       # (Q,3)
    src_flux: np.ndarray       # (Q,)
    lmn: np.ndarray            # (P,3) pixel grid
    times: np.ndarray          # (T,) seconds from mid-observation

    def positions(self, step: int) -> np.ndarray:
        lat = math.radians(self.cfg.latitude_deg)
        return enu_to_celestial(self.enu, lat, EARTH_OMEGA * self.times[step])


def observation(cfg: SimConfig) -> Observation:
    lat = math.radians(cfg.latitude_deg)
    basis = uvw_basis(0.0, lat)
    enu = antenna_layout_enu(cfg)
    dirs, flux = sky(cfg, basis)
    lmn = make_lmn_grid(cfg.image_size, math.radians(cfg.fov_deg))
    t = (np.arange(cfg.n_steps) - (cfg.n_steps - 1) / 2.0) * cfg.dt_s
    return Observation(cfg, basis, enu, dirs, flux, lmn, t)


def keep_masks(cfg: SimConfig) -> np.ndarray:
    """(T, N) bool: antennas kept (not flagged) per step."""
    n, t = cfg.n_antenna, cfg.n_steps
    if cfg.keep is None:
        return np.ones((t, n), dtype=bool)
    rng = np.random.default_rng(cfg.seed + 2000)
    masks = np.zeros((t, n), dtype=bool)
    for s in range(t):
        k = int(rng.integers(cfg.keep[0], cfg.keep[1] + 1))
        masks[s, rng.choice(n, size=k, replace=False)] = True
    return masks


def visibilities(obs: Observation, steps: Sequence[int], device="cpu", dtype=None,
                 masks: Optional[np.ndarray] = None, wl: Optional[float] = None,
                 noise_key: int = 0) -> Tuple[torch.Tensor, torch.Tensor]:
    """S (len(steps), N, N) and positions xyz (len(steps), N, 3) for the given steps at
    wavelength wl (default cfg.wl). Noise X ~ CN(0, sigma^2), E = (X + X^H)/2; diagonal
    zeroed; flagged antennas become zero rows/columns. noise_key separates the noise of
    the frequency channels of one step."""
    cfg = obs.cfg
    wl = cfg.wl if wl is None else wl
    if dtype is None:
        dtype = torch.complex128 if cfg.double else torch.complex64
    rdtype = torch.float64 if dtype == torch.complex128 else torch.float32
    n = cfg.n_antenna
    xyz = np.stack([obs.positions(s) for s in steps])                       # (B,N,3) float64
    xyz_t = torch.from_numpy(xyz).to(device)
    dirs = torch.from_numpy(obs.src_dirs).to(device)
    flux = torch.from_numpy(obs.src_flux).to(device)
    # phase (B,Q,N) in float64, then complex
    ph = (2 * math.pi / wl) * torch.einsum("qc,bnc->bqn", dirs, xyz_t)
    a = torch.polar(torch.ones_like(ph), ph)                                 # exp(+i 2pi/wl r.p)
    s = torch.einsum("bqi,q,bqj->bij", a.conj(), flux.to(a.dtype), a)     # sum_q I_q e^{-i..(p_i-p_j)}
    g = torch.Generator(device=device)
    g.manual_seed(cfg.seed * 1000003 + int(steps[0]) + 7919 * int(noise_key))
    sig = cfg.noise_sigma / math.sqrt(2.0)
    xr = torch.randn((len(steps), n, n), generator=g, device=device, dtype=torch.float64) * sig
    xi = torch.randn((len(steps), n, n), generator=g, device=device, dtype=torch.float64) * sig
    x = torch.complex(xr, xi)
    s = s + 0.5 * (x + x.conj().transpose(1, 2))
    s.diagonal(dim1=1, dim2=2).zero_()
    if masks is not None:
        m = torch.from_numpy(masks[list(steps)]).to(device).to(torch.float64)
        s = s * (m[:, :, None] * m[:, None, :])
    return s.to(dtype), xyz_t.to(rdtype if rdtype == torch.float64 else torch.float64)


def antenna_uvw(obs: Observation, xyz: np.ndarray) -> np.ndarray:
    """(N,3) antenna coordinates in the UVW frame (float64)."""
    return xyz @ obs.basis


def baseline_uvw(obs: Observation, xyz: np.ndarray) -> np.ndarray:
    """(N^2, 3) float32 baseline uvw with k = i + j N <-> p_i - p_j
    (python/bipp/frame.py:75-89)."""
    au = antenna_uvw(obs, xyz)
    b = au[:, None, :] - au[None, :, :]          # b[i, j] = U_i - U_j
    return np.ascontiguousarray(b.transpose(1, 0, 2).reshape(-1, 3)).astype(np.float32)
