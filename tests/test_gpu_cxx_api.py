"""GPU: the bipp C++ API shell (include/bipp/*.hpp over libbipp_b200.so) compiled with
g++ and called like the reference's own test calls eigh_gram, on the reference's LOFAR
test input; results compared to the reference's outputs."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, golden

pytestmark = pytest.mark.gpu


def test_cxx_api_eigh_gram_lofar(tmp_path):
    g = golden("lofar.npz")
    k = 0
    s, w, xyz = g["s"][k], g["w"][k], g["xyz"][k]
    nA, nB = w.shape
    np.asfortranarray(s, dtype=np.complex128).T.tofile(tmp_path / "s.bin")
    np.asfortranarray(w, dtype=np.complex128).T.tofile(tmp_path / "w.bin")
    np.asfortranarray(xyz, dtype=np.float64).T.tofile(tmp_path / "xyz.bin")
    exe = tmp_path / "api_check"
    libdir = os.path.join(ROOT, "bipp_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cxx", "api_check.cpp"),
                    "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L" + libdir,
                    "-lbipp_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    r = subprocess.run([str(exe), str(tmp_path), str(nA), str(nB), repr(float(g["wl"]))], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    dref = g["d_f64"][k]
    vref = g["v_f64"][k]
    pref = (vref * dref) @ vref.conj().T
    for tag, dt, ct, tol in (("f32", np.float32, np.complex64, 1e-5), ("f64", np.float64, np.complex128, 1e-10)):
        d = np.fromfile(tmp_path / f"d_{tag}.bin", dtype=dt)
        v = np.fromfile(tmp_path / f"v_{tag}.bin", dtype=ct).reshape((nB, nA)).T
        meta = np.fromfile(tmp_path / f"meta_{tag}.bin", dtype=np.float64)
        assert int(meta[0]) == int(g[f"nred_{tag}"][k])
        assert abs(meta[1] - float(g[f"scale_{tag}"][k])) <= 1e-6 * meta[1]
        assert np.abs(d - dref).max() <= tol * np.abs(dref).max()
        p = (v.astype(np.complex128) * d) @ v.astype(np.complex128).conj().T
        assert np.abs(p - pref).max() <= (1e-4 if tag == "f32" else 1e-9) * np.abs(pref).max()


def test_cxx_api_image_synthesis_two_ranks(tmp_path):
    """bipp::image_synthesis of the C++ API under Communicator::world() with two ranks
    (two processes on this GPU, images summed into rank 0 over TCP; their kernels never
    wait on each other) equals the single-rank call, to 1e-5 relative L2 per image; 7
    samples, so the ranks image 4 and 3 (src/image_synthesis.cpp:75-80)."""
    import socket

    from bipp_b200 import simulate as sim
    from oracle import bluebild as bb

    cfg = sim.config_c1(n_antenna=40, n_steps=7)
    obs = sim.observation(cfg)
    s, xyz = sim.visibilities(obs, list(range(7)))
    s, xyz = s.numpy(), xyz.numpy()
    N, ns = cfg.n_antenna, 7
    V, D, UVW, SC = [], [], [], []
    for k in range(ns):
        v, d, nr, sc = bb.eigh_gram(cfg.wl, s[k], np.eye(N), xyz[k])
        V.append(np.asfortranarray(v, dtype=np.complex64).T.reshape(-1))
        D.append(d.astype(np.float32))
        au = xyz[k] @ obs.basis
        UVW.append(np.asfortranarray((au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3),
                                     dtype=np.float32).T.reshape(-1))
        SC.append(sc)
    np.concatenate(V).tofile(tmp_path / "v.bin")
    np.concatenate(D).tofile(tmp_path / "d.bin")
    np.concatenate(UVW).tofile(tmp_path / "uvw.bin")
    np.full(ns, cfg.wl, np.float32).tofile(tmp_path / "wl.bin")
    np.array(SC, np.float32).tofile(tmp_path / "scale.bin")
    mid = np.median(np.concatenate(D)[np.concatenate(D) > 0])
    ev = np.stack([np.stack([d * ((d > 0) & (d <= mid)) for d in D]), np.stack([d * (d > mid) for d in D])])
    ev.astype(np.float32).tofile(tmp_path / "ev.bin")
    rng = np.random.default_rng(4)
    npix = 500
    lm = rng.uniform(-0.05, 0.05, (npix, 2))
    lmn = np.column_stack([lm, np.sqrt(1 - (lm ** 2).sum(1))]).astype(np.float32)
    np.asfortranarray(lmn).T.tofile(tmp_path / "lmn.bin")
    exe = tmp_path / "multirank_check"
    libdir = os.path.join(ROOT, "bipp_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", os.path.join(ROOT, "tests", "cxx", "multirank_check.cpp"),
                    "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L" + libdir,
                    "-lbipp_b200", "-Wl,-rpath," + libdir, "-o", str(exe)], check=True)
    args = [str(tmp_path), str(ns), str(N), str(N), str(npix)]
    env1 = dict(os.environ, RANK="0", WORLD_SIZE="1")
    r = subprocess.run([str(exe)] + args + [str(tmp_path / "one.bin")], env=env1, capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    procs = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", MASTER_ADDR="127.0.0.1",
                   BIPP_B200_REDUCE_PORT=str(port), BIPP_B200_REDUCE_TIMEOUT="120")
        procs.append(subprocess.Popen([str(exe)] + args + [str(tmp_path / f"two_{rank}.bin")], env=env,
                                      stderr=subprocess.PIPE, text=True))
    for p in procs:
        _, err = p.communicate(timeout=300)
        assert p.returncode == 0, err
    one = np.fromfile(tmp_path / "one.bin", dtype=np.float32).reshape(2, npix).astype(np.float64)
    two = np.fromfile(tmp_path / "two_0.bin", dtype=np.float32).reshape(2, npix).astype(np.float64)
    assert not (tmp_path / "two_1.bin").exists()
    for t in range(2):
        assert np.linalg.norm(two[t] - one[t]) <= 1e-5 * np.linalg.norm(one[t]), t
