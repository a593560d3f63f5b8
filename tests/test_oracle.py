"""CPU: the numpy restatement (oracle/bluebild.py) pinned against the reference's own
outputs (golden fixtures made by running the compiled reference sources), and against
the compiled reference directly when it is available in this container."""
import numpy as np
import pytest

from conftest import golden, nonfinite_cases
from oracle import bluebild as bb
from oracle import ref


def _pair_product(v, d):
    return (v * d) @ v.conj().T


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_lofar_eigh_gram(prec):
    g = golden("lofar.npz")
    for k in range(g["s"].shape[0]):
        v, d, nr, sc = bb.eigh_gram(float(g["wl"]), g["s"][k], g["w"][k], g["xyz"][k])
        assert nr == int(g[f"nred_{prec}"][k]) == 54
        assert abs(sc - float(g[f"scale_{prec}"][k])) <= 1e-6 * sc
        dref = g[f"d_{prec}"][k]
        tol = 1e-12 if prec == "f64" else 2e-5
        assert np.abs(d - dref).max() <= tol * np.abs(dref).max()
        p = _pair_product(v, d)
        pref = _pair_product(g[f"v_{prec}"][k].astype(np.complex128), dref.astype(np.float64))
        assert np.abs(p - pref).max() <= (1e-11 if prec == "f64" else 1e-4) * np.abs(pref).max()


def test_lofar_virtual_vis():
    g = golden("lofar.npz")
    for k in range(g["s"].shape[0]):
        d = g["d_f64"][k]
        n_eig = int(g["n_eig"])
        for lv, (lo, hi) in enumerate(g["intervals"]):
            dl = d.copy()
            dl[:n_eig] *= (dl[:n_eig] >= lo) & (dl[:n_eig] <= hi)
            dl[n_eig:] = 0
            vv = bb.virtual_vis(float(g["scale_f64"][k]), dl, g["v_f64"][k])
            ref_vv = g["vv_f64"][k][lv]
            assert np.abs(vv - ref_vv).max() <= 1e-12 * max(np.abs(ref_vv).max(), 1e-300)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_synthetic_eigh_and_flagging(prec):
    g = golden("synth_eig.npz")
    n = g["s"].shape[1]
    for k in range(g["s"].shape[0]):
        dt = np.float64 if prec == "f64" else np.float32
        v, d, nr, sc = bb.eigh_gram(float(g["wl"]), g["s"][k], np.eye(n), g["xyz"][k], dtype=dt)
        assert nr == int(g[f"nred_{prec}"][k])
        assert abs(sc - float(g[f"scale_{prec}"][k])) <= 1e-6 * sc
        dref = g[f"d_{prec}"][k]
        tol = 1e-12 if prec == "f64" else 2e-5
        assert np.abs(d - dref).max() <= tol * np.abs(dref).max()
        v2, d2, nr2, sc2 = bb.eigh(float(g["wl"]), g["s"][k], np.eye(n), dtype=dt)
        assert nr2 == int(g[f"snred_{prec}"][k])
        assert np.abs(d2 - g[f"sd_{prec}"][k]).max() <= tol * np.abs(g[f"sd_{prec}"][k]).max()
    # step 1 has four flagged antennas
    assert int(g["nred_f64"][1]) == n - 4


def test_nuft_sum_oracle():
    g = golden("nuft.npz")
    out = bb.nuft_sum(float(g["alpha"]), g["vals"], g["u"], g["v"], g["w"], g["x"], g["y"], g["z"])
    assert np.abs(out - g["out64"]).max() <= 1e-10 * np.abs(g["out64"]).max()


@pytest.mark.parametrize("prec", ["f32", "f64"])
@pytest.mark.parametrize("n", [1, 100, 4000])
def test_partition_oracle(n, prec):
    g = golden("partition.npz")
    dt = np.float32 if prec == "f32" else np.float64
    pm, gb, gs = bb.partition_grid([2, 3, 4], g[f"x_{n}_{prec}"], g[f"y_{n}_{prec}"], g[f"z_{n}_{prec}"], dtype=dt)
    assert (pm == g[f"permut_{n}_{prec}"]).all()
    assert (gb == g[f"begin_{n}_{prec}"]).all()
    assert (gs == g[f"size_{n}_{prec}"]).all()


def test_partition_invariants():
    """The reference's DomainPartition test invariants (tests/test_domain_partition.cpp:24-94)."""
    rng = np.random.default_rng(3)
    for n in (1, 100, 4000):
        x, y, z = rng.uniform(-5, 10, n), rng.uniform(2, 20, n), rng.uniform(100, 5000, n)
        pm, gb, gs = bb.partition_grid([2, 3, 4], x, y, z)
        cover = np.zeros(n, bool)
        for b, s in zip(gb, gs):
            cover[int(b):int(b + s)] = True
        assert cover.all()
        assert sorted(pm.tolist()) == list(range(n))
        for c, dims in ((x, 2), (y, 3), (z, 4)):
            spacing = (c.max() - c.min()) / dims
            srt = np.empty(n)
            srt[pm.astype(np.int64)] = c
            for b, s in zip(gb, gs):
                if s:
                    seg = srt[int(b):int(b + s)]
                    assert seg.max() - seg.min() <= spacing + 1e-12


def test_energy_levels_and_filters():
    d = np.array([-1.0, 0.0, 0.5, 2.0, 9.0])
    assert np.allclose(bb.level_eigenvalues(d, 0.0, 1.0), [0, 0, 0.5, 0, 0])
    assert np.allclose(bb.apply_filter("std", d), np.sign(d))
    assert np.allclose(bb.apply_filter("sqrt", d), np.sign(d) * np.sqrt(np.abs(d)))
    inv = bb.apply_filter("inv", d)
    assert inv[1] == 0 and np.isclose(inv[3], 0.5)
    iv = bb.centroid_to_intervals(np.array([10.0, 1.0, 0.1]), 0.0, 100.0)
    assert np.allclose(iv[:, 0], [5.5, 0.55, 0.0]) and np.allclose(iv[:, 1], [100.0, 5.5, 0.55])


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
def test_restatement_vs_compiled_reference_random():
    rng = np.random.default_rng(11)
    n = 24
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = a @ a.conj().T / n
    np.fill_diagonal(s, 0)
    s[:, 5] = 0
    s[5, :] = 0
    xyz = rng.uniform(-50, 50, (n, 3))
    w = np.eye(n)
    v_r, d_r, nr_r, sc_r = ref.eigh_gram(2.0, s, w, xyz)
    v_o, d_o, nr_o, sc_o = bb.eigh_gram(2.0, s, w, xyz)
    assert nr_r == nr_o == n - 1 and sc_r == sc_o
    assert np.abs(d_r - d_o).max() <= 1e-12 * np.abs(d_r).max()
    g_r = ref.gram_matrix(w, xyz, 2.0)
    assert np.abs(g_r - bb.gram_matrix(w, xyz, 2.0)).max() <= 1e-14


@pytest.mark.parametrize("fn", ["eigh_gram", "eigh"])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_nonfinite_entries(fn, dtype):
    """A NaN antenna is dropped like a zero antenna; a NaN/Inf in a kept entry of the lower
    triangle raises EigensolverError; one above the diagonal is never read."""
    xyz, zero_ant, nan_ant, upper, bad = nonfinite_cases()
    n = zero_ant.shape[0]
    call = (lambda s: bb.eigh_gram(2.0, s, np.eye(n), xyz, dtype=dtype)) if fn == "eigh_gram" else \
        (lambda s: bb.eigh(2.0, s, np.eye(n), dtype=dtype))
    vz, dz, nz, sz = call(zero_ant)
    vn, dn, nn, sn = call(nan_ant)
    assert nz == nn == n - 1 and sz == sn
    assert np.array_equal(dz, dn) and np.array_equal(vz, vn)
    assert call(upper)[2] == n
    for s in bad.values():
        with pytest.raises(bb.EigensolverError):
            call(s)


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
@pytest.mark.parametrize("fn", ["eigh_gram", "eigh"])
def test_nonfinite_entries_match_compiled_reference(fn):
    xyz, zero_ant, nan_ant, upper, bad = nonfinite_cases()
    n = zero_ant.shape[0]
    for dt in (np.float64, np.float32):
        if fn == "eigh_gram":
            r = lambda s: ref.eigh_gram(2.0, s, np.eye(n), xyz, dtype=dt)  # noqa: E731
            o = lambda s: bb.eigh_gram(2.0, s, np.eye(n), xyz, dtype=dt)  # noqa: E731
        else:
            r = lambda s: ref.eigh(2.0, s, np.eye(n), dtype=dt)  # noqa: E731
            o = lambda s: bb.eigh(2.0, s, np.eye(n), dtype=dt)  # noqa: E731
        for s in (nan_ant, upper):
            vr, dr, nr, sr = r(s)
            vo, do, no, so = o(s)
            assert nr == no and abs(sr - so) <= 1e-6 * sr
            assert np.abs(dr - do).max() <= (1e-12 if dt == np.float64 else 2e-5) * np.abs(dr).max()
        for s in bad.values():
            with pytest.raises(RuntimeError, match="BippError 6"):
                r(s)
            with pytest.raises(bb.EigensolverError):
                o(s)


def test_levels_and_filters_match_reference_python():
    """Energy-level intervals (k-means, seed 42), the centroid-to-interval rule (also for
    centroids in arbitrary order) and the five eigenvalue filters, unbounded and through
    the level bounds, against the reference's own Python run on the same inputs
    (tests/golden/levels.npz); the oracle and the host-side estimator of the package both."""
    from bipp_b200 import parameter_estimator as pe

    g = golden("levels.npz")
    for k in range(len(g["case_n"])):
        args = (int(g["case_n"][k]), float(g["case_sigma"][k]), str(g["case_func"][k]), float(g["case_lo"][k]),
                float(g["case_hi"][k]), g["d_all"])
        want = g[f"intervals_{k}"]
        for got in (bb.infer_intervals(*args), pe.infer_intervals(*args)):
            assert got.shape == want.shape
            assert np.allclose(got, want, rtol=1e-12, atol=0)
    k = 0
    while f"centroid_{k}" in g.files:
        for fn in (bb.centroid_to_intervals, pe.centroid_to_intervals):
            assert np.array_equal(fn(g[f"centroid_{k}"], 0.0, 100.0), g[f"centroid_intervals_{k}"])
        k += 1
    d = g["filter_d"]
    for name in g["filters"]:
        name = str(name)
        assert np.array_equal(bb.apply_filter(name, d), g[f"filter_{name}"])
        assert np.array_equal(bb.level_eigenvalues(d, -0.5, 2.0, name), g[f"filter_{name}_bounded"])
    with pytest.raises(ValueError):
        bb.infer_intervals(2, 1.0, "log", -1.0, np.inf, g["d_all"])
    with pytest.raises(ValueError):
        pe.infer_intervals(2, 1.0, "log", -1.0, np.inf, g["d_all"])


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
@pytest.mark.parametrize("seed", [1, 2, 3])
def test_restatement_vs_compiled_reference_beamformed(seed):
    """Random beamformed problems (complex W, nBeam < nAntenna, flagged beams): eigh_gram,
    eigh, the Gram matrix, virtual visibilities and the direct sum of the restatement
    against the compiled reference, in FP64 (FP32 for the direct sum as well)."""
    rng = np.random.default_rng(100 + seed)
    n_ant, n_beam = 30, 18
    w = (rng.standard_normal((n_ant, n_beam)) + 1j * rng.standard_normal((n_ant, n_beam))) / np.sqrt(n_ant)
    xyz = rng.uniform(-40, 40, (n_ant, 3))
    a = rng.standard_normal((n_beam, n_beam)) + 1j * rng.standard_normal((n_beam, n_beam))
    s = a @ a.conj().T / n_beam
    s[:, 2 + seed] = s[2 + seed, :] = 0
    wl = 1.5 + 0.5 * seed
    g_r, g_o = ref.gram_matrix(w, xyz, wl), bb.gram_matrix(w, xyz, wl)
    assert np.abs(g_r - g_o).max() <= 1e-12 * np.abs(g_r).max()
    v_r, d_r, nr_r, sc_r = ref.eigh_gram(wl, s, w, xyz)
    v_o, d_o, nr_o, sc_o = bb.eigh_gram(wl, s, w, xyz)
    assert nr_r == nr_o == n_beam - 1 and sc_r == sc_o
    assert np.abs(d_r - d_o).max() <= 1e-10 * np.abs(d_r).max()
    p_r, p_o = _pair_product(v_r, d_r), _pair_product(v_o, d_o)
    assert np.abs(p_r - p_o).max() <= 1e-9 * np.abs(p_r).max()
    v2_r, d2_r, nr2_r, _ = ref.eigh(wl, s, w)
    v2_o, d2_o, nr2_o, _ = bb.eigh(wl, s, w)
    assert nr2_r == nr2_o and np.abs(d2_r - d2_o).max() <= 1e-12 * np.abs(d2_r).max()
    p2_r, p2_o = _pair_product(v2_r, d2_r), _pair_product(v2_o, d2_o)   # v = W_red X
    assert np.abs(p2_r - p2_o).max() <= 1e-10 * np.abs(p2_r).max()
    # one level: the upper half of the spectrum, as the reference's level mask
    dl = d_r * (d_r >= np.median(d_r[:nr_r]))
    vv_r, vv_o = ref.virtual_vis(sc_r, dl, v_r), bb.virtual_vis(sc_r, dl, v_r)
    assert np.abs(vv_r - vv_o).max() <= 1e-12 * np.abs(vv_r).max()
    # direct sum of those virtual visibilities onto random pixels
    au = xyz @ rng.standard_normal((3, 3))
    uvw = (au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3) * (2 * np.pi / wl)
    pix = rng.uniform(-0.1, 0.1, (64, 3))
    vals = vv_r.reshape(-1, order="F")
    for dt, tol in ((np.float64, 1e-10), (np.float32, 1e-5)):
        out_r = ref.nuft_sum(1.0, vals, uvw[:, 0], uvw[:, 1], uvw[:, 2], pix[:, 0], pix[:, 1], pix[:, 2], dtype=dt)
        out_o = bb.nuft_sum(1.0, vals, uvw[:, 0], uvw[:, 1], uvw[:, 2], pix[:, 0], pix[:, 1], pix[:, 2])
        assert np.abs(out_r - out_o).max() <= tol * np.abs(out_o).max()


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
def test_lofar_image_oracle_vs_compiled_reference():
    """The FP64 image oracle (bb.image_synthesis, which the GPU image tests compare against)
    against the compiled reference's own pieces on the reference's LOFAR test input, in
    the flow of tests/test_nufft_synthesis_lofar.cpp:86-233: eigh_gram<float> per sample,
    the level mask with its index cut at n_eig_int (:112-124), virtual_vis<double>, the
    exact sum nuft_sum<double> that the NUFFT approximates, 1/nSamples. The pixel grid of
    the missing output file is replaced by a 24 x 24 grid of direction cosines."""
    g = golden("lofar.npz")
    wl, n_eig, intervals = float(g["wl"]), int(g["n_eig"]), g["intervals"]
    l, m = np.meshgrid(np.linspace(-0.05, 0.05, 24), np.linspace(-0.04, 0.06, 24))
    l, m = l.ravel(), m.ravel()
    lmn = np.stack([l, m, np.sqrt(1 - l ** 2 - m ** 2)], 1)
    steps, want = [], np.zeros((lmn.shape[0], len(intervals)))
    for k in range(g["s"].shape[0]):
        v, d, nr, sc = ref.eigh_gram(wl, g["s"][k], g["w"][k], g["xyz"][k], dtype=np.float32)
        assert nr == n_eig
        steps.append(dict(uvw=g["uvw"][k], v=v, d=d, scale=sc, wl=wl))
        uvw = g["uvw"][k].astype(np.float64) * (2 * np.pi / wl)
        for lv, (lo, hi) in enumerate(intervals):
            dl = d.astype(np.float64)
            dl[:n_eig] *= (dl[:n_eig] >= lo) & (dl[:n_eig] <= hi)
            dl[n_eig:] = 0
            vv = ref.virtual_vis(sc, dl, v.astype(np.complex128)).reshape(-1, order="F")
            want[:, lv] += ref.nuft_sum(1.0, vv, uvw[:, 0], uvw[:, 1], uvw[:, 2], lmn[:, 0], lmn[:, 1], lmn[:, 2])
    want /= len(steps)
    got = bb.image_synthesis(steps, intervals, lmn)
    for lv in range(len(intervals)):
        assert np.abs(want[:, lv]).max() > 0
        assert np.abs(got[:, lv] - want[:, lv]).max() <= 1e-9 * np.abs(want[:, lv]).max()


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_flag_threshold_matches_compiled_reference(dtype):
    """Antennas whose only entries sit at the flag threshold (|s|^2 vs eps for eigh_gram,
    |Re|, |Im| vs eps for eigh; eps of the working precision, src/eigensolver.cpp:57-76,
    148-166): kept or dropped exactly as by the reference, with the same 1/nVis."""
    rng = np.random.default_rng(3)
    n = 16
    eps = float(np.finfo(dtype).eps)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = a @ a.conj().T / n
    xyz = rng.uniform(-30, 30, (n, 3))
    factors = (0.5, 0.999, 1.0, 1.001, 2.0)
    sg, se = s.copy(), s.copy()
    for k, f in zip(range(3, 3 + len(factors)), factors):
        sg[k, :] = sg[:, k] = 0
        sg[k, 0] = np.sqrt(f * eps)          # |s|^2 = f eps (up to rounding in the precision)
        sg[0, k] = np.conj(sg[k, 0])
        se[k, :] = se[:, k] = 0
        se[k, 1] = complex(0.0, f * eps)     # |Im| = f eps
        se[1, k] = np.conj(se[k, 1])
    r = ref.eigh_gram(2.0, sg, np.eye(n), xyz, dtype=dtype)
    o = bb.eigh_gram(2.0, sg, np.eye(n), xyz, dtype=dtype)
    assert r[2] == o[2] and abs(r[3] - o[3]) <= 1e-6 * r[3]
    r = ref.eigh(2.0, se, np.eye(n), dtype=dtype)
    o = bb.eigh(2.0, se, np.eye(n), dtype=dtype)
    assert r[2] == o[2] and abs(r[3] - o[3]) <= 1e-6 * r[3]
    assert n - len(factors) < o[2] < n


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
def test_partition_matches_compiled_reference_property():
    """DomainPartition::grid of the restatement equals the compiled reference bit for bit
    on random grids, sizes and value ranges (degenerate axes and duplicates included)."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=120, deadline=None, database=None)
    @given(st.integers(0, 300), st.lists(st.integers(1, 5), min_size=3, max_size=3), st.integers(0, 2 ** 31),
           st.sampled_from([np.float32, np.float64]), st.booleans())
    def check(n, dims, seed, dt, degenerate):
        rng = np.random.default_rng(seed)
        x = rng.uniform(-5, 10, n).astype(dt)
        y = (np.full(n, 3.0) if degenerate else rng.uniform(2, 20, n)).astype(dt)
        z = np.round(rng.uniform(100, 5000, n), 0).astype(dt)      # repeated values
        pm_r, gb_r, gs_r = ref.partition_grid(dims, x, y, z, dtype=dt)
        pm_o, gb_o, gs_o = bb.partition_grid(dims, x, y, z, dtype=dt)
        assert np.array_equal(pm_r, pm_o) and np.array_equal(gb_r, gb_o) and np.array_equal(gs_r, gs_o)

    check()


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_all_flagged_step_raises_like_compiled_reference(dtype):
    """Every row and column flagged: the reference's LAPACK call gets a 0 x 0 problem with
    leading dimension 0 and rejects it (EigensolverError); one non-zero pair keeps two."""
    n = 6
    xyz = np.random.default_rng(1).uniform(0, 10, (n, 3))
    for fn_r, fn_o in ((lambda s: ref.eigh_gram(2.0, s, np.eye(n), xyz, dtype=dtype),
                        lambda s: bb.eigh_gram(2.0, s, np.eye(n), xyz, dtype=dtype)),
                       (lambda s: ref.eigh(2.0, s, np.eye(n), dtype=dtype),
                        lambda s: bb.eigh(2.0, s, np.eye(n), dtype=dtype))):
        with pytest.raises(RuntimeError, match="BippError 6"):
            fn_r(np.zeros((n, n)))
        with pytest.raises(bb.EigensolverError):
            fn_o(np.zeros((n, n)))
        s = np.zeros((n, n), complex)
        s[2, 1] = s[1, 2] = 1.0
        assert fn_r(s)[2] == fn_o(s)[2] == 2


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
def test_eigensolvers_match_compiled_reference_property():
    """Random flag patterns (dropped antennas, isolated entries, entries near the flag
    threshold, diagonal-only antennas) and both precisions: the restatement's nReduced,
    1/nVis and eigenvalues equal the compiled reference's, eigh_gram and eigh."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=80, deadline=None, database=None)
    @given(st.integers(2, 14), st.integers(0, 2 ** 31), st.sampled_from([np.float32, np.float64]))
    def check(n, seed, dt):
        rng = np.random.default_rng(seed)
        eps = float(np.finfo(dt).eps)
        a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
        s = a @ a.conj().T / n
        kind = rng.integers(0, 4, n)          # 0 keep, 1 drop, 2 one tiny entry, 3 diagonal only
        for k in range(n):
            if kind[k] == 0:
                continue
            s[k, :] = 0
            s[:, k] = 0
            if kind[k] == 2:
                j = int(rng.integers(0, n))
                val = np.sqrt(eps) * rng.uniform(0.5, 2.0)
                s[max(j, k), min(j, k)] = val
                s[min(j, k), max(j, k)] = val
            elif kind[k] == 3:
                s[k, k] = rng.uniform(0.5, 2.0)
        xyz = rng.uniform(-20, 20, (n, 3))
        for fr, fo in ((lambda m: ref.eigh_gram(2.0, m, np.eye(n), xyz, dtype=dt),
                        lambda m: bb.eigh_gram(2.0, m, np.eye(n), xyz, dtype=dt)),
                       (lambda m: ref.eigh(2.0, m, np.eye(n), dtype=dt),
                        lambda m: bb.eigh(2.0, m, np.eye(n), dtype=dt))):
            try:
                r = fr(s)
            except RuntimeError:
                with pytest.raises(bb.EigensolverError):
                    fo(s)
                continue
            o = fo(s)
            assert r[2] == o[2]
            assert abs(r[3] - o[3]) <= 1e-6 * max(r[3], 1e-30)
            tol = 1e-10 if dt == np.float64 else 1e-4
            assert np.abs(r[1] - o[1]).max() <= tol * max(np.abs(r[1]).max(), 1e-30)

    check()


@pytest.mark.skipif(not ref.available(), reason="compiled reference not built in this environment")
def test_gram_and_virtual_vis_match_compiled_reference_property():
    """Random beamforming matrices, positions, wavelengths and level eigenvalues (zeros,
    negatives): Gram matrix and virtual visibilities of the restatement equal the compiled
    reference's (FP64)."""
    from hypothesis import given, settings, strategies as st

    @settings(max_examples=60, deadline=None, database=None)
    @given(st.integers(1, 12), st.integers(1, 12), st.integers(0, 2 ** 31), st.floats(0.2, 5.0))
    def check(n_ant, n_beam, seed, wl):
        rng = np.random.default_rng(seed)
        w = rng.standard_normal((n_ant, n_beam)) + 1j * rng.standard_normal((n_ant, n_beam))
        xyz = rng.uniform(-30, 30, (n_ant, 3))
        g_r, g_o = ref.gram_matrix(w, xyz, wl), bb.gram_matrix(w, xyz, wl)
        assert np.abs(g_r - g_o).max() <= 1e-12 * max(np.abs(g_r).max(), 1e-300)
        v = rng.standard_normal((n_ant, n_beam)) + 1j * rng.standard_normal((n_ant, n_beam))
        d = rng.standard_normal(n_beam) * (rng.uniform(size=n_beam) > 0.3)
        sc = float(rng.uniform(1e-3, 1.0))
        vv_r, vv_o = ref.virtual_vis(sc, d, v), bb.virtual_vis(sc, d, v)
        assert np.abs(vv_r - vv_o).max() <= 1e-12 * max(np.abs(vv_r).max(), 1e-300)

    check()


def test_mlp_oracle_gradient_by_finite_differences():
    """The numpy statement of the rank predictor's network (oracle/mlp.py): its
    backpropagated gradient equals central differences of its loss (FP64) on random
    parameters of every layer."""
    from oracle import mlp as om

    rng = np.random.default_rng(5)
    n = 37
    X = rng.standard_normal((n, om.F))
    y = rng.uniform(0, 1, n)
    model = np.concatenate([rng.standard_normal(om.F) * 0.1, rng.uniform(0.5, 2.0, om.F),
                            rng.standard_normal(om.N_PARAMS - 2 * om.F) * 0.2])
    loss, g = om.loss_and_gradient(model, X, y)
    assert np.all(g[:om.OFF["W1"]] == 0)
    idx = np.concatenate([rng.choice(np.arange(lo, hi), 6, replace=False) for lo, hi in
                          ((om.OFF["W1"], om.OFF["b1"]), (om.OFF["b1"], om.OFF["W2"]), (om.OFF["W2"], om.OFF["b2"]),
                           (om.OFF["b2"], om.OFF["W3"]), (om.OFF["W3"], om.OFF["b3"]))] + [[om.OFF["b3"]]])
    h = 1e-6
    for i in idx:
        mp, mm = model.copy(), model.copy()
        mp[i] += h
        mm[i] -= h
        fd = (om.loss_and_gradient(mp, X, y)[0] - om.loss_and_gradient(mm, X, y)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_mlp_oracle_features_statement():
    """The numpy feature statement on a small Hermitian matrix: scale-free (a scaled
    matrix gives the same features except the threshold), the largest diagonal
    magnitudes first, the largest rows' share of the Frobenius norm and the probe moments
    in their ranges."""
    from oracle import mlp as om

    rng = np.random.default_rng(6)
    a = rng.standard_normal((40, 40)) + 1j * rng.standard_normal((40, 40))
    C = (a + a.conj().T) / 2
    f = om.features(C, 0.0)
    f2 = om.features(7.0 * C, 0.0)
    assert np.allclose(f, f2)
    assert np.all(np.diff(f[:32]) <= 0)
    assert 0 < f[63] <= 1.0
    # the probe moments: t2 / f^2 is an unbiased estimate of 1; t4 / f^4 <= 1
    assert 0.5 < f[60] < 1.5 and 0 < f[47] <= 1.0
    assert np.isclose(f[35], np.count_nonzero(C.diagonal().real > 0) / 40)
