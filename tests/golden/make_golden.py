"""Generate the golden fixtures of tests/golden/ by running the reference's own CPU code.

Run in a container where the reference tree and oracle/_ref/libbipp_ref.so exist:

    make -C oracle REF=<reference tree> && python tests/golden/make_golden.py <reference tree>

Outputs (compressed .npz, a few hundred KB in total):
  lofar.npz      inputs of the reference's test data tests/data/lofar_input.json (2 samples,
                 55 antennas, beamformed W) and the outputs of the reference's
                 eigh_gram<float/double> (src/eigensolver.cpp:129-225) and virtual_vis
                 (src/host/virtual_vis.cpp:19-73) for the two intervals of that test
                 (tests/test_nufft_synthesis_lofar.cpp:112-124).
  synth_eig.npz  seeded synthetic steps (60 antennas, one with flagged antennas), reference
                 eigh_gram / eigh outputs in both precisions, virtual_vis per level.
  nuft.npz       reference nuft_sum<double/float> (src/host/kernels/nuft_sum.cpp:9-31) on a
                 seeded small problem.
  partition.npz  reference DomainPartition::grid (src/host/domain_partition.hpp:35-101) on the
                 seeded distributions of tests/test_domain_partition.cpp:102-131 (numpy RNG).
  frame.npz      the reference's own python/bipp/frame.py (uvw_basis, make_grids,
                 reshape_uvw: the UVW frame, the pixel grid and the baseline order) on a
                 few field centres, grid sizes and random UVW.
  levels.npz     the reference's own Python energy-level estimator and eigenvalue filters
                 (python/bipp/parameter_estimator.py:18-105, python/bipp/filter.py:7-51)
                 on seeded eigenvalue spectra, loaded from the reference's source files.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref  # noqa: E402
from bipp_b200 import simulate as sim  # noqa: E402


def lofar(refdir: str):
    d = json.load(open(os.path.join(refdir, "tests", "data", "lofar_input.json")))
    out = {"wl": d["wl"], "n_eig": d["n_eig_int"], "intervals": np.array(d["intervals_int"])}
    xyzs, ss, ws, uvws = [], [], [], []
    for it in d["data"]:
        xyzs.append(np.array(it["xyz"]).T)
        ss.append((np.array(it["s_real"]) + 1j * np.array(it["s_imag"])).T)
        ws.append((np.array(it["w_real"]) + 1j * np.array(it["w_imag"])).T)
        # the test rescales uvw back by wl / 2 pi (tests/test_nufft_synthesis_lofar.cpp:144-150)
        uvws.append(np.array(it["uvw"]).T * (d["wl"] / (2 * np.pi)))
    out["xyz"] = np.array(xyzs)
    out["s"] = np.array(ss)
    out["w"] = np.array(ws)
    out["uvw"] = np.array(uvws, dtype=np.float32)
    for prec, dt in (("f32", np.float32), ("f64", np.float64)):
        vs, ds, nrs, scs, vvs = [], [], [], [], []
        for k in range(len(ss)):
            v, dd, nr, sc = ref.eigh_gram(d["wl"], ss[k], ws[k], xyzs[k], dtype=dt)
            vs.append(v)
            ds.append(dd)
            nrs.append(nr)
            scs.append(sc)
            lv = []
            for lo, hi in d["intervals_int"]:
                dl = dd.copy()
                n_eig = d["n_eig_int"]
                dl[:n_eig] *= (dl[:n_eig] >= lo) & (dl[:n_eig] <= hi)
                dl[n_eig:] = 0
                lv.append(ref.virtual_vis(sc, dl, v, dtype=dt))
            vvs.append(lv)
        out[f"v_{prec}"] = np.array(vs)
        out[f"d_{prec}"] = np.array(ds)
        out[f"nred_{prec}"] = np.array(nrs)
        out[f"scale_{prec}"] = np.array(scs)
        out[f"vv_{prec}"] = np.array(vvs)
        # the same samples with identity beamforming (W = I over the 55 stations): the
        # input of the batched eigh_gram, which takes W = I
        eye = [ref.eigh_gram(d["wl"], ss[k], np.eye(ss[k].shape[0]), xyzs[k], dtype=dt) for k in range(len(ss))]
        out[f"eye_v_{prec}"] = np.array([e[0] for e in eye])
        out[f"eye_d_{prec}"] = np.array([e[1] for e in eye])
        out[f"eye_nred_{prec}"] = np.array([e[2] for e in eye])
        out[f"eye_scale_{prec}"] = np.array([e[3] for e in eye])
    np.savez_compressed(os.path.join(HERE, "lofar.npz"), **out)


def synth_eig():
    cfg = sim.config_c1(n_steps=3)
    obs = sim.observation(cfg)
    masks = np.ones((3, cfg.n_antenna), dtype=bool)
    masks[1, [3, 17, 40, 41]] = False  # one step with flagged antennas
    s, xyz = sim.visibilities(obs, [0, 1, 2], masks=masks)
    s = s.numpy()
    xyz = xyz.numpy()
    n = cfg.n_antenna
    w = np.eye(n)
    out = {"wl": cfg.wl, "s": s, "xyz": xyz}
    intervals = np.array([[0.0, 50.0], [50.0, np.finfo(np.float32).max]])
    out["intervals"] = intervals
    for prec, dt in (("f32", np.float32), ("f64", np.float64)):
        res = {k: [] for k in ("v", "d", "nred", "scale", "vv", "sv", "sd", "snred", "sscale")}
        for k in range(3):
            v, dd, nr, sc = ref.eigh_gram(cfg.wl, s[k], w, xyz[k], dtype=dt)
            res["v"].append(v)
            res["d"].append(dd)
            res["nred"].append(nr)
            res["scale"].append(sc)
            res["vv"].append([ref.virtual_vis(sc, dd * ((dd >= lo) & (dd <= hi)), v, dtype=dt) for lo, hi in intervals])
            v2, d2, nr2, sc2 = ref.eigh(cfg.wl, s[k], w, dtype=dt)
            res["sv"].append(v2)
            res["sd"].append(d2)
            res["snred"].append(nr2)
            res["sscale"].append(sc2)
        for key, val in res.items():
            out[f"{key}_{prec}"] = np.array(val)
    np.savez_compressed(os.path.join(HERE, "synth_eig.npz"), **out)


def nuft():
    rng = np.random.default_rng(7)
    m, p = 500, 300
    vals = rng.standard_normal(m) + 1j * rng.standard_normal(m)
    u, v, w = rng.uniform(-1, 1, (3, m)) * np.array([[3000.0], [3000.0], [200.0]])
    x, y = rng.uniform(-0.15, 0.15, (2, p))
    z = np.sqrt(1 - x ** 2 - y ** 2)
    alpha = 2 * np.pi / 2.0
    out64 = ref.nuft_sum(alpha, vals, u, v, w, x, y, z, dtype=np.float64)
    out32 = ref.nuft_sum(alpha, vals, u, v, w, x, y, z, dtype=np.float32)
    np.savez_compressed(os.path.join(HERE, "nuft.npz"), alpha=alpha, vals=vals, u=u, v=v, w=w, x=x, y=y, z=z,
                        out64=out64, out32=out32)


def partition():
    out = {}
    rng = np.random.default_rng(42)
    for n in (1, 100, 4000):
        x = rng.uniform(-5.0, 10.0, n)
        y = rng.uniform(2.0, 20.0, n)
        z = rng.uniform(100.0, 5000.0, n)
        for prec, dt in (("f32", np.float32), ("f64", np.float64)):
            pm, gb, gs = ref.partition_grid([2, 3, 4], x.astype(dt), y.astype(dt), z.astype(dt), dtype=dt)
            out[f"x_{n}_{prec}"] = x.astype(dt)
            out[f"y_{n}_{prec}"] = y.astype(dt)
            out[f"z_{n}_{prec}"] = z.astype(dt)
            out[f"permut_{n}_{prec}"] = pm
            out[f"begin_{n}_{prec}"] = gb
            out[f"size_{n}_{prec}"] = gs
    np.savez_compressed(os.path.join(HERE, "partition.npz"), **out)


def _load_reference_levels(refdir: str):
    """The reference's parameter_estimator.py and filter.py, executed from its source tree.
    Their package imports (bipp.pybipp, bipp.statistics, bipp.gram, bipp.imot_tools) are
    stubbed with empty modules: the functions used here need only numpy and scikit-learn."""
    import importlib.util
    import types

    names = ["bipp", "bipp.imot_tools", "bipp.imot_tools.math", "bipp.imot_tools.math.linalg",
             "bipp.imot_tools.util", "bipp.imot_tools.util.argcheck", "bipp.statistics", "bipp.gram", "bipp.pybipp",
             "bipp.filter"]
    saved = {k: sys.modules.get(k) for k in names}
    stubs = {k: types.ModuleType(k) for k in names}
    for k, m in stubs.items():
        if "." in k:
            parent, child = k.rsplit(".", 1)
            setattr(stubs[parent], child, m)
    sys.modules.update(stubs)

    def load(modname, rel):
        spec = importlib.util.spec_from_file_location(modname, os.path.join(refdir, rel))
        m = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(m)
        return m

    try:
        filt = load("bipp.filter", os.path.join("python", "bipp", "filter.py"))
        sys.modules["bipp.filter"] = filt
        stubs["bipp"].filter = filt
        pe = load("bipp_reference_parameter_estimator", os.path.join("python", "bipp", "parameter_estimator.py"))
    finally:
        for k, m in saved.items():
            if m is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = m
    return pe, filt


# (n_level, sigma, cluster_func, d_min, d_max) cases of infer_intervals
LEVEL_CASES = [(4, 1.0, "log", 0.0, np.inf), (8, 0.95, "log", 0.0, 1e6), (3, 0.9, "log", 1e-3, np.inf),
               (1, 1.0, "log", 0.0, np.inf), (4, 1.0, "none", -50.0, 1e4), (2, 0.99, "none", 0.0, np.inf)]
FILTERS = ["lsq", "std", "sqrt", "inv", "inv_sqrt"]


def levels(refdir: str):
    pe, filt = _load_reference_levels(refdir)
    rng = np.random.default_rng(7)
    # a spectrum like a time step's: a few strong source eigenvalues, a lognormal bulk,
    # zeros (padding of flagged antennas) and small negative noise eigenvalues
    d_all = np.concatenate([rng.lognormal(3.0, 1.5, 40), rng.lognormal(-1.0, 1.0, 1500), np.zeros(60),
                            -rng.lognormal(-3.0, 0.5, 200)])
    rng.shuffle(d_all)
    out = {"d_all": d_all, "case_n": np.array([c[0] for c in LEVEL_CASES]),
           "case_sigma": np.array([c[1] for c in LEVEL_CASES]), "case_func": np.array([c[2] for c in LEVEL_CASES]),
           "case_lo": np.array([c[3] for c in LEVEL_CASES]), "case_hi": np.array([c[4] for c in LEVEL_CASES]),
           "filters": np.array(FILTERS)}
    for k, (n, sigma, f, lo, hi) in enumerate(LEVEL_CASES):
        out[f"intervals_{k}"] = pe.infer_intervals(n, sigma, f, lo, hi, d_all)
    # centroids in arbitrary order (the interval rule indexes the sorted centroids with
    # the original positions)
    for k, c in enumerate([np.array([10.0, 1.0, 0.1]), np.array([3.0, 10.0, 1.0, 0.1]), np.array([0.5, 7.0]),
                           np.array([2.0])]):
        out[f"centroid_{k}"] = c
        out[f"centroid_intervals_{k}"] = pe.centroid_to_intervals(c, 0.0, 100.0)
    d = np.array([-4.0, -0.25, 0.0, 0.25, 1.0, 9.0])
    out["filter_d"] = d
    for name in FILTERS:
        out[f"filter_{name}"] = filt.apply_filter(name, d.copy())
        out[f"filter_{name}_bounded"] = filt.Filter(name, -0.5, 2.0)(d.copy())
    np.savez_compressed(os.path.join(HERE, "levels.npz"), **out)


def frame(refdir: str):
    """frame.py loaded from the reference's source with astropy.coordinates stubbed: the
    functions only read a field centre's lon/lat (radians) and unit vector."""
    import importlib.util
    import types

    saved = {k: sys.modules.get(k) for k in ("astropy", "astropy.coordinates")}
    astropy = types.ModuleType("astropy")
    coords = types.ModuleType("astropy.coordinates")
    coords.SkyCoord = object
    astropy.coordinates = coords
    sys.modules.update({"astropy": astropy, "astropy.coordinates": coords})
    try:
        spec = importlib.util.spec_from_file_location("bipp_reference_frame",
                                                      os.path.join(refdir, "python", "bipp", "frame.py"))
        fr = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(fr)
    finally:
        for k, m in saved.items():
            if m is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = m

    def centre(lon, lat):
        xyz = np.array([np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)])
        return types.SimpleNamespace(data=types.SimpleNamespace(lon=types.SimpleNamespace(rad=lon),
                                                                lat=types.SimpleNamespace(rad=lat)),
                                     cartesian=types.SimpleNamespace(xyz=types.SimpleNamespace(value=xyz)))

    out = {}
    cases = [(0.0, -0.5235987755982988), (1.2, 0.3), (4.0, -1.1)]
    out["centres"] = np.array(cases)
    for k, (lon, lat) in enumerate(cases):
        out[f"basis_{k}"] = fr.uvw_basis(centre(lon, lat))
    grids = [(8, 0.2), (33, 0.28), (64, 0.05)]
    out["grids"] = np.array(grids)
    for k, (n, fov) in enumerate(grids):
        lmn, _ = fr.make_grids(int(n), fov, centre(*cases[0]))
        out[f"lmn_{k}"] = lmn
    rng = np.random.default_rng(9)
    au = rng.standard_normal((7, 3)) * 100.0     # antenna UVW coordinates
    out["antenna_uvw"] = au
    out["uvw_reshaped"] = fr.reshape_uvw(au[:, None, :] - au[None, :, :])   # UVW[i, j] = U_i - U_j
    np.savez_compressed(os.path.join(HERE, "frame.npz"), **out)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <reference tree>")
    refdir = sys.argv[1]
    lofar(refdir)
    synth_eig()
    nuft()
    partition()
    levels(refdir)
    frame(refdir)
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))
