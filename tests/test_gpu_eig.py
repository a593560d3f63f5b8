"""GPU parity of the eigensolver entry points against the reference's own outputs
(golden fixtures from the compiled reference) and the FP64 oracle.

Tolerances: FP64 entry points agree with the reference's zhegv to 1e-10 relative;
FP32 entry points agree with the FP64 reference to 1e-5 relative on eigenvalues
(normwise, max|d - d_ref| / max|d_ref|) and 1e-4 on V diag(d) V^H."""
import numpy as np
import pytest

from conftest import golden, nonfinite_cases
from oracle import bluebild as bb
from oracle import ref

pytestmark = pytest.mark.gpu


def _prod(v, d):
    v = v.astype(np.complex128)
    return (v * d.astype(np.float64)) @ v.conj().T


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_lofar_eigh_gram_general_w(ctx, prec):
    import bipp_b200 as bipp

    g = golden("lofar.npz")
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    for k in range(g["s"].shape[0]):
        v, d, nr, sc = bipp.eigh_gram_full(dt(g["wl"]), g["s"][k].astype(ct), g["w"][k].astype(ct),
                                           g["xyz"][k].astype(dt), ctx=ctx)
        assert nr == int(g[f"nred_{prec}"][k])
        assert abs(sc - float(g[f"scale_{prec}"][k])) <= 1e-6 * sc
        dref = g["d_f64"][k]
        tol_d, tol_p = (1e-10, 1e-9) if prec == "f64" else (1e-5, 1e-4)
        assert _rel(d, dref) <= tol_d
        assert np.all(d[nr:] == 0)
        assert _rel(_prod(v, d), _prod(g["v_f64"][k], dref)) <= tol_p


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_synthetic_eigh_gram_with_flagging(ctx, prec):
    import bipp_b200 as bipp

    g = golden("synth_eig.npz")
    n = g["s"].shape[1]
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    for k in range(g["s"].shape[0]):
        v, d, nr, sc = bipp.eigh_gram_full(dt(g["wl"]), g["s"][k].astype(ct), np.eye(n, dtype=ct),
                                           g["xyz"][k].astype(dt), ctx=ctx)
        assert nr == int(g[f"nred_{prec}"][k])
        assert abs(sc - float(g[f"scale_{prec}"][k])) <= 1e-6 * sc
        tol_d, tol_p = (1e-10, 1e-9) if prec == "f64" else (1e-5, 1e-4)
        assert _rel(d, g["d_f64"][k]) <= tol_d
        assert _rel(_prod(v, d), _prod(g["v_f64"][k], g["d_f64"][k])) <= tol_p
        # flagged antennas give zero rows of v
        if nr < n:
            flagged = np.abs(g["s"][k]).sum(0) == 0
            assert np.all(v[flagged] == 0)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_synthetic_eigh_standard(ctx, prec):
    import bipp_b200 as bipp

    g = golden("synth_eig.npz")
    n = g["s"].shape[1]
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    for k in range(g["s"].shape[0]):
        v, d, nr, sc = bipp.eigh(dt(g["wl"]), g["s"][k].astype(ct), np.eye(n, dtype=ct), ctx=ctx, full=True)
        assert nr == int(g[f"snred_{prec}"][k])
        tol_d, tol_p = (1e-10, 1e-9) if prec == "f64" else (1e-5, 1e-4)
        assert _rel(d, g["sd_f64"][k]) <= tol_d
        assert _rel(_prod(v, d), _prod(g["sv_f64"][k], g["sd_f64"][k])) <= tol_p


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_lofar_eigh_general_w(ctx, prec):
    """The standard eigh (no Gram matrix) with the LOFAR input's complex beamforming W:
    eigenvalues and the beamformed V diag(d) V^H (v = W_red X) against the oracle, which
    is pinned to the compiled reference on beamformed problems."""
    import bipp_b200 as bipp

    g = golden("lofar.npz")
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    tol_d, tol_p = (1e-10, 1e-9) if prec == "f64" else (1e-5, 1e-4)
    for k in range(g["s"].shape[0]):
        v, d, nr, sc = bipp.eigh(dt(g["wl"]), g["s"][k].astype(ct), g["w"][k].astype(ct), ctx=ctx, full=True)
        vr, dr, nrr, scr = bb.eigh(float(dt(g["wl"])), g["s"][k].astype(ct), g["w"][k].astype(ct), dtype=dt)
        assert nr == nrr and abs(sc - scr) <= 1e-6 * scr
        assert _rel(d, dr) <= tol_d
        assert _rel(_prod(v, d), _prod(vr, dr)) <= tol_p


def test_eigenvector_g_orthonormality(ctx):
    import bipp_b200 as bipp

    g = golden("synth_eig.npz")
    n = g["s"].shape[1]
    s, xyz = g["s"][0], g["xyz"][0]
    v, d, nr, sc = bipp.eigh_gram_full(float(g["wl"]), s, np.eye(n), xyz, ctx=ctx)
    G = bb.gram_matrix(np.eye(n), xyz, float(g["wl"]))
    x = v[:, :nr]
    assert np.abs(x.conj().T @ G @ x - np.eye(nr)).max() < 1e-9
    assert np.abs(s @ x - G @ x * d[:nr]).max() < 1e-9 * np.abs(s).max()


def _per_eig_rel(d, dref, lo=0.0):
    """Largest per-eigenvalue relative error over the eigenvalues of dref above lo (the
    level range [0, inf) of the benchmark), edges within 1e-6 max|dref| of lo left out."""
    sel = dref > lo + 1e-6 * np.abs(dref).max()
    return float((np.abs(d[sel] - dref[sel]) / np.abs(dref[sel])).max()) if sel.any() else 0.0


@pytest.mark.parametrize("n", [64, 200, 300, 512, 768])
def test_larger_sizes_against_fp64_oracle(ctx, n):
    """FP32 GPU eigensolve at N up to 768 against scipy FP64, with random flagging: the
    unblocked tridiagonalisation (N = 64), and the blocked one with 256 (N = 200), 512
    (N = 300, 512) and 1024 (N = 768) threads per matrix. Per eigenvalue (over the
    positive eigenvalues, the ones the energy levels image) the relative error is at most
    1e-5 or twice that of the reference's own FP32 path (eigh_gram<float>, chegv) on the
    same input, whichever is larger."""
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    cfg = sim.config_c2(n_antenna=n, n_steps=2, n_src=min(200, n // 2))
    obs = sim.observation(cfg)
    masks = np.ones((2, n), dtype=bool)
    rng = np.random.default_rng(n)
    masks[1, rng.choice(n, size=n // 5, replace=False)] = False
    s, xyz = sim.visibilities(obs, [0, 1], masks=masks)
    s, xyz = s.numpy(), xyz.numpy()
    for k in range(2):
        v, d, nr, sc = bipp.eigh_gram_full(np.float32(cfg.wl), s[k].astype(np.complex64), np.eye(n, dtype=np.complex64),
                                           xyz[k].astype(np.float32), ctx=ctx)
        vo, do, nro, sco = bb.eigh_gram(cfg.wl, s[k].astype(np.complex64).astype(np.complex128), np.eye(n),
                                        xyz[k].astype(np.float32).astype(np.float64))
        assert nr == nro
        assert _rel(d, do) <= 1e-5
        assert _rel(_prod(v, d), _prod(vo, do)) <= 1e-4
        if ref.available():
            _, d32, _, _ = ref.eigh_gram(np.float32(cfg.wl), s[k].astype(np.complex64), np.eye(n, dtype=np.complex64),
                                         xyz[k].astype(np.float32), dtype=np.float32)
            gpu, cpu32 = _per_eig_rel(d, do), _per_eig_rel(d32, do)
            print(f"n={n} step {k}: per-eigenvalue rel. error GPU {gpu:.2e}, reference FP32 {cpu32:.2e}")
            assert gpu <= max(1e-5, 2 * cpu32), (gpu, cpu32)


def test_batched_eigh_gram_matches_single(ctx):
    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    cfg = sim.config_c2(n_antenna=96, n_steps=5, n_src=40, keep=(70, 96))
    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    s, xyz = sim.visibilities(obs, list(range(5)), masks=masks)
    s, xyz = s.numpy(), xyz.numpy()
    wl = np.full(5, cfg.wl, dtype=np.float32)
    v, d, nred, scale = bipp.eigh_gram_batched(wl, s, xyz, ctx=ctx)
    for k in range(5):
        vs, ds, nrs, scs = bipp.eigh_gram_full(np.float32(cfg.wl), s[k], np.eye(96, dtype=np.complex64),
                                               xyz[k].astype(np.float32), ctx=ctx)
        assert nred[k] == nrs == masks[k].sum()
        assert abs(scale[k] - scs) <= 1e-7 * scs
        assert _rel(d[k], ds) <= 1e-6
        assert _rel(_prod(v[k], d[k]), _prod(vs, ds)) <= 1e-5


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batched_eigh_gram_against_compiled_reference(ctx, prec):
    """The batched eigh_gram (W = I) against the reference's own eigh_gram outputs: the
    three golden 60-antenna steps (one with flagged antennas) in one batch, and the two
    LOFAR samples (55 stations, the reference's test input) with identity beamforming.
    FP32: eigenvalues 1e-5 relative to zhegv (normwise), V diag(d) V^H 1e-4, nBeamReduced
    and 1/nVis of eigh_gram<float>; FP64: 1e-10 and 1e-9."""
    import bipp_b200 as bipp

    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    tol_d, tol_p = (1e-10, 1e-9) if prec == "f64" else (1e-5, 1e-4)
    for name, pre in (("synth_eig.npz", ""), ("lofar.npz", "eye_")):
        g = golden(name)
        B = g["s"].shape[0]
        v, d, nred, scale = bipp.eigh_gram_batched(np.full(B, g["wl"], dtype=dt), g["s"].astype(ct),
                                                   g["xyz"].astype(dt), ctx=ctx,
                                                   precision="double" if prec == "f64" else "single")
        for k in range(B):
            assert nred[k] == int(g[f"{pre}nred_{prec}"][k])
            assert abs(scale[k] - float(g[f"{pre}scale_{prec}"][k])) <= 1e-6 * scale[k]
            dref = g[f"{pre}d_f64"][k]
            assert _rel(d[k], dref) <= tol_d
            assert _rel(_prod(v[k], d[k]), _prod(g[f"{pre}v_f64"][k], dref)) <= tol_p


def test_all_flagged_step(ctx):
    """Every row and column flagged: the reference hands LAPACK a 0 x 0 problem with
    leading dimension 0, which LAPACK rejects, and throws EigensolverError
    (src/eigensolver.cpp:172-223, src/host/lapack_api.hpp:133); so do these entry points."""
    import bipp_b200 as bipp

    n = 16
    with pytest.raises(bipp.EigensolverError):
        bipp.eigh_gram_full(2.0, np.zeros((n, n), np.complex128), np.eye(n), np.random.rand(n, 3), ctx=ctx)
    # the context is still usable
    xyz, zero_ant, _, _, _ = nonfinite_cases()
    assert bipp.eigh_gram_full(2.0, zero_ant, np.eye(24), xyz, ctx=ctx)[2] == 23


def test_invalid_gram_raises_eigensolver_error(ctx):
    """A non-finite antenna position makes a Cholesky pivot of G NaN: the FP64 Cholesky
    reports it and the call raises EigensolverError, as LAPACK ?potrf/?hegv does in the
    reference (src/host/lapack_api.hpp:133)."""
    import bipp_b200 as bipp

    n = 8
    rng = np.random.default_rng(0)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = a @ a.conj().T
    xyz = rng.uniform(0, 100, (n, 3))
    xyz[3, 0] = np.nan
    with pytest.raises(bipp.EigensolverError):
        bipp.eigh_gram(2.0, s, np.eye(n), xyz, ctx=ctx)


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("fn", ["eigh_gram", "eigh"])
def test_nonfinite_entries_as_reference(ctx, prec, fn):
    """Non-finite visibilities behave as in the reference (the oracle is pinned to the
    compiled reference on these cases): a NaN antenna is dropped like a zero antenna, a
    NaN above the diagonal is never read, a NaN/Inf in a kept entry of the lower triangle
    raises EigensolverError, and the context stays usable after the error."""
    import bipp_b200 as bipp

    xyz, zero_ant, nan_ant, upper, bad = nonfinite_cases()
    n = zero_ant.shape[0]
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    eye = np.eye(n, dtype=ct)
    xyz_t = xyz.astype(dt)
    if fn == "eigh_gram":
        call = lambda s: bipp.eigh_gram_full(dt(2.0), s.astype(ct), eye, xyz_t, ctx=ctx)  # noqa: E731
        orc = lambda s: bb.eigh_gram(2.0, s.astype(ct), np.eye(n), xyz_t.astype(np.float64))  # noqa: E731
    else:
        call = lambda s: bipp.eigh(dt(2.0), s.astype(ct), eye, ctx=ctx, full=True)  # noqa: E731
        orc = lambda s: bb.eigh(2.0, s.astype(ct), np.eye(n))  # noqa: E731
    tol_d, tol_p = (1e-10, 1e-9) if prec == "f64" else (1e-5, 1e-4)
    for s in (zero_ant, nan_ant, upper):
        v, d, nr, sc = call(s)
        vr, dr, nrr, scr = orc(s)
        assert nr == nrr and abs(sc - scr) <= 1e-6 * scr
        assert _rel(d, dr) <= tol_d
        assert _rel(_prod(v, d), _prod(vr, dr)) <= tol_p
    for name, s in bad.items():
        with pytest.raises(bipp.EigensolverError):
            call(s)
    assert call(zero_ant)[2] == n - 1


def test_nonfinite_entries_batched(ctx):
    """The batched eigh_gram: a NaN antenna step equals its zero-antenna twin, and one step
    with a NaN in a kept entry fails the call with EigensolverError."""
    import bipp_b200 as bipp

    xyz, zero_ant, nan_ant, upper, bad = nonfinite_cases()
    xyz3 = np.stack([xyz] * 3).astype(np.float32)
    wl = np.full(3, 2.0, dtype=np.float32)
    s = np.stack([zero_ant, nan_ant, upper]).astype(np.complex64)
    v, d, nred, scale = bipp.eigh_gram_batched(wl, s, xyz3, ctx=ctx)
    assert nred[0] == nred[1] == 23 and nred[2] == 24 and scale[0] == scale[1]
    assert _rel(d[1], d[0]) <= 1e-6
    assert _rel(_prod(v[1], d[1]), _prod(v[0], d[0])) <= 1e-5
    s[1] = bad["lower"].astype(np.complex64)
    with pytest.raises(bipp.EigensolverError):
        bipp.eigh_gram_batched(wl, s, xyz3, ctx=ctx)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_gram_matrix(ctx, prec):
    import bipp_b200 as bipp

    g = golden("lofar.npz")
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    G = bipp.gram_matrix(g["xyz"][0].astype(dt), g["w"][0].astype(ct), dt(g["wl"]), ctx=ctx)
    Gr = bb.gram_matrix(g["w"][0].astype(ct), g["xyz"][0].astype(dt), float(dt(g["wl"])))
    assert _rel(G, Gr) <= (1e-12 if prec == "f64" else 1e-5)


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_virtual_vis(ctx, prec):
    import bipp_b200 as bipp

    g = golden("lofar.npz")
    dt, ct = (np.float64, np.complex128) if prec == "f64" else (np.float32, np.complex64)
    n_eig = int(g["n_eig"])
    for k in range(2):
        d = g[f"d_{prec}"][k]
        for lv, (lo, hi) in enumerate(g["intervals"]):
            dl = d.copy()
            dl[:n_eig] *= (dl[:n_eig] >= lo) & (dl[:n_eig] <= hi)
            dl[n_eig:] = 0
            vv = bipp.virtual_vis(dt(g[f"scale_{prec}"][k]), dl.astype(dt), g[f"v_{prec}"][k].astype(ct), ctx=ctx)
            ref_vv = g[f"vv_{prec}"][k][lv]
            scale = max(np.abs(ref_vv).max(), 1e-30)
            assert np.abs(vv - ref_vv).max() <= (1e-12 if prec == "f64" else 1e-5) * scale


def test_bounded_barrier_wait_reports_timeout(ctx):
    """The bounded wait of the tensor-core kernels on a barrier that nothing completes
    (bipp_selftest_wait_timeout, a short spin limit): it gives up, the call fails with
    BIPP_GPU_ERROR (GPUError), and the context still runs the tensor-core eigensolver."""
    import ctypes as C

    import bipp_b200 as bipp
    from bipp_b200._lib import check

    out = C.c_int(0)
    with pytest.raises(bipp.GPUError):
        check(ctx._lib.bipp_selftest_wait_timeout(ctx.handle, 2000, C.byref(out)))
    assert out.value == 1
    g = golden("synth_eig.npz")
    n = g["s"].shape[1]
    v, d, nr, sc = bipp.eigh_gram_full(np.float32(g["wl"]), g["s"][0].astype(np.complex64), np.eye(n, dtype=np.complex64),
                                       g["xyz"][0].astype(np.float32), ctx=ctx)
    assert _rel(d, g["d_f64"][0]) <= 1e-5
