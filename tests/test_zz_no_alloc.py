"""GPU: the allocation-free eigh_gram entry point (bipp_eigh_gram_noalloc_s) against the
regular one (bipp_eigh_gram_s), called twice in a row through the C ABI, against the
compiled reference's eigh_gram (golden fixture), and with the device's free memory
unchanged by a call.

Callers that cannot let a library allocate device memory (a host framework whose caching
allocator owns the device memory, a real-time loop that must not block on cudaFree) use
that entry point; its intermediates live in a fixed-size file-scope device array, so two
consecutive calls also check that stale contents of that array do not leak into the next
result. Tolerances as in the eigensolver parity tests: eigenvalues 1e-6 relative,
V diag(d) V^H 1e-5 relative, between the two GPU entry points; 1e-5 and 1e-4 against the
reference's FP64 zhegv."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _case(n, seed, flagged=()):
    from bipp_b200 import simulate as sim

    cfg = sim.config_c2(n_antenna=n, n_steps=1, n_src=min(40, n // 2), seed=seed, extent_m=5000.0)
    obs = sim.observation(cfg)
    masks = np.ones((1, n), dtype=bool)
    masks[0, list(flagged)] = False
    s, xyz = sim.visibilities(obs, [0], masks=masks)
    return cfg.wl, s.numpy()[0].astype(np.complex64), xyz.numpy()[0]


class _Buffers:
    """Device inputs and outputs of one call, allocated before the call."""

    def __init__(self, wl, s, xyz):
        import torch

        n = s.shape[0]
        dev = torch.device("cuda", 0)
        self.n, self.wl = n, wl
        self.s = torch.from_numpy(np.ascontiguousarray(s.T)).to(dev)      # column-major S
        self.x = torch.from_numpy(np.ascontiguousarray(xyz.T)).to(dev)    # column-major xyz (n x 3)
        self.d = torch.empty(n, dtype=torch.float32, device=dev)
        self.v = torch.empty((n, n), dtype=torch.complex64, device=dev)   # column-major: v[c, a]
        self.nr = torch.empty(1, dtype=torch.int32, device=dev)
        self.sc = torch.empty(1, dtype=torch.float32, device=dev)
        self.info = torch.empty(1, dtype=torch.int32, device=dev)
        self.stream = torch.cuda.current_stream(dev)

    def call(self, lib):
        from bipp_b200._lib import check

        n = self.n
        check(lib.bipp_eigh_gram_noalloc_s(0, C.c_void_p(self.stream.cuda_stream), np.float32(self.wl), n,
                                           C.c_void_p(self.s.data_ptr()), n, C.c_void_p(self.x.data_ptr()), n,
                                           C.c_void_p(self.d.data_ptr()), C.c_void_p(self.v.data_ptr()), n,
                                           C.c_void_p(self.nr.data_ptr()), C.c_void_p(self.sc.data_ptr()),
                                           C.c_void_p(self.info.data_ptr())))


def _noalloc(lib, wl, s, xyz):
    import torch

    b = _Buffers(wl, s, xyz)
    b.call(lib)
    torch.cuda.synchronize()
    return (b.v.cpu().numpy().T, b.d.cpu().numpy(), int(b.nr.item()), float(b.sc.item()), int(b.info.item()))


def _prod(v, d):
    v = v.astype(np.complex128)
    return (v * d.astype(np.float64)) @ v.conj().T


def test_noalloc_matches_regular_entry_point_twice():
    import bipp_b200 as bipp
    from bipp_b200 import _lib

    lib = _lib.load()
    ctx = bipp.Context("GPU", device=0)
    cases = [_case(96, 11, flagged=(3, 50, 77)), _case(40, 12)]   # second call: smaller, stale data behind it
    for wl, s, xyz in cases:
        v1, d1, nr1, sc1 = bipp.eigh_gram_full(np.float32(wl), s, np.eye(s.shape[0], dtype=np.complex64),
                                               xyz.astype(np.float32), ctx=ctx)
        v2, d2, nr2, sc2, info = _noalloc(lib, wl, s, xyz.astype(np.float32).astype(np.float64))
        assert info == 0
        assert nr2 == nr1
        assert abs(sc2 - sc1) <= 1e-7 * sc1
        assert np.abs(d2 - d1).max() <= 1e-6 * np.abs(d1).max()
        p1, p2 = _prod(v1, d1), _prod(v2, d2)
        assert np.abs(p2 - p1).max() <= 1e-5 * np.abs(p1).max()
    ctx.close()


def test_noalloc_against_compiled_reference_fixture():
    """The golden steps (60 antennas, one with flagged antennas, W = I) against the
    reference's own eigh_gram outputs: eigenvalues of zhegv to 1e-5 relative, V diag(d) V^H
    to 1e-4, nBeamReduced and 1/nVis of eigh_gram<float>."""
    from bipp_b200 import _lib
    from conftest import golden

    lib = _lib.load()
    g = golden("synth_eig.npz")
    for k in range(g["s"].shape[0]):
        v, d, nr, sc, info = _noalloc(lib, float(g["wl"]), g["s"][k].astype(np.complex64),
                                      g["xyz"][k].astype(np.float32).astype(np.float64))
        assert info == 0
        assert nr == int(g["nred_f32"][k])
        assert abs(sc - float(g["scale_f32"][k])) <= 1e-6 * sc
        dref = g["d_f64"][k]
        assert np.abs(d - dref).max() <= 1e-5 * np.abs(dref).max()
        p, pref = _prod(v, d), _prod(g["v_f64"][k], dref)
        assert np.abs(p - pref).max() <= 1e-4 * np.abs(pref).max()


def test_noalloc_allocates_no_device_memory():
    """With its buffers allocated and one call made (the first call may load device code),
    a further call leaves the device's free memory (cudaMemGetInfo) unchanged, and the
    caller's current device is the same after the call."""
    import torch

    from bipp_b200 import _lib

    lib = _lib.load()
    wl, s, xyz = _case(96, 13, flagged=(5,))
    b = _Buffers(wl, s, xyz.astype(np.float32).astype(np.float64))
    b.call(lib)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(0)[0]
    dev0 = torch.cuda.current_device()
    for _ in range(3):
        b.call(lib)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(0)[0] == free0
    assert torch.cuda.current_device() == dev0
    assert int(b.info.item()) == 0 and int(b.nr.item()) == 95


def test_noalloc_rejects_sizes_above_the_maximum():
    from bipp_b200 import _lib

    lib = _lib.load()
    n = 200
    buf = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.bipp_eigh_gram_noalloc_s(0, None, np.float32(2.0), n, buf, n, buf, n, buf, buf, n, buf, buf, buf)
    assert rc == 3
    assert b"BIPP_NOALLOC_MAX_ANTENNA" in lib.bipp_last_error()


def test_noalloc_nonfinite_entries():
    """Non-finite visibilities as in the reference: a NaN antenna is dropped like a zero
    antenna (info 0), a NaN in a kept entry of the lower triangle gives info 1 (the
    reference's EigensolverError), and the next call is unaffected."""
    from bipp_b200 import _lib
    from conftest import nonfinite_cases

    lib = _lib.load()
    xyz, zero_ant, nan_ant, upper, bad = nonfinite_cases()
    xyz = xyz.astype(np.float32).astype(np.float64)
    vz, dz, nz, sz, iz = _noalloc(lib, 2.0, zero_ant.astype(np.complex64), xyz)
    vn, dn, nn, sn, inn = _noalloc(lib, 2.0, nan_ant.astype(np.complex64), xyz)
    assert iz == inn == 0 and nz == nn == zero_ant.shape[0] - 1 and sz == sn
    assert np.abs(dn - dz).max() <= 1e-6 * np.abs(dz).max()
    assert np.abs(_prod(vn, dn) - _prod(vz, dz)).max() <= 1e-5 * np.abs(_prod(vz, dz)).max()
    assert _noalloc(lib, 2.0, bad["lower"].astype(np.complex64), xyz)[4] == 1
    assert _noalloc(lib, 2.0, zero_ant.astype(np.complex64), xyz)[4] == 0
