"""GPU: the allocation-free eigh_gram entry point (bipp_eigh_gram_noalloc_s) against the
regular one (bipp_eigh_gram_s), called twice in a row through the C ABI.

Callers that cannot let a library allocate device memory (a host framework whose caching
allocator owns the device memory, a real-time loop that must not block on cudaFree) use
that entry point; its intermediates live in a fixed-size file-scope device array, so two
consecutive calls also check that stale contents of that array do not leak into the next
result. Tolerances as in the eigensolver parity tests: eigenvalues 1e-6 relative,
V diag(d) V^H 1e-5 relative, between the two GPU entry points."""
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


def _noalloc(lib, wl, s, xyz):
    import torch

    n = s.shape[0]
    dev = torch.device("cuda", 0)
    s_d = torch.from_numpy(np.ascontiguousarray(s.T)).to(dev)      # column-major S
    x_d = torch.from_numpy(np.ascontiguousarray(xyz.T)).to(dev)    # column-major xyz (n x 3)
    d_d = torch.empty(n, dtype=torch.float32, device=dev)
    v_d = torch.empty((n, n), dtype=torch.complex64, device=dev)   # column-major: v_d[c, a]
    nr_d = torch.empty(1, dtype=torch.int32, device=dev)
    sc_d = torch.empty(1, dtype=torch.float32, device=dev)
    info_d = torch.empty(1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    from bipp_b200._lib import check

    check(lib.bipp_eigh_gram_noalloc_s(0, C.c_void_p(stream.cuda_stream), np.float32(wl), n, C.c_void_p(s_d.data_ptr()),
                                       n, C.c_void_p(x_d.data_ptr()), n, C.c_void_p(d_d.data_ptr()),
                                       C.c_void_p(v_d.data_ptr()), n, C.c_void_p(nr_d.data_ptr()),
                                       C.c_void_p(sc_d.data_ptr()), C.c_void_p(info_d.data_ptr())))
    torch.cuda.synchronize()
    return (v_d.cpu().numpy().T, d_d.cpu().numpy(), int(nr_d.item()), float(sc_d.item()), int(info_d.item()))


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
