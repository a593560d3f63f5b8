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
