"""Test infrastructure only: ctypes access to the reference's own CPU code.

``oracle/_ref/libbipp_ref.so`` is built by ``oracle/Makefile`` from the
reference's unmodified sources (src/eigensolver.cpp, src/host/gram_matrix.cpp,
src/host/virtual_vis.cpp, src/host/kernels/nuft_sum.cpp, and the header-only
src/host/domain_partition.hpp) plus ``oracle/ref_shim.cpp``. It pins the numpy
restatement in ``oracle/bluebild.py`` and is the CPU baseline of
``bench.py --impl reference``. Only tests, ``__graft_entry__.smoke`` and the
CPU-baseline leg of ``bench.py`` may import this module.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libbipp_ref.so")
_lib = None

_sz = C.c_size_t
_p = C.c_void_p


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference oracle library missing: {LIB_PATH} (run make -C oracle)")
        L = C.CDLL(LIB_PATH)
        for prec, fl in (("f32", C.c_float), ("f64", C.c_double)):
            fn = getattr(L, f"ref_eigh_gram_{prec}")
            fn.argtypes = [fl, _sz, _sz, _p, _sz, _p, _sz, _p, _sz, _p, _p, _sz, C.POINTER(_sz), C.POINTER(fl)]
            fn.restype = C.c_int
            fn = getattr(L, f"ref_eigh_{prec}")
            fn.argtypes = [fl, _sz, _sz, _p, _sz, _p, _sz, _p, _p, _sz, C.POINTER(_sz), C.POINTER(fl)]
            fn.restype = C.c_int
            fn = getattr(L, f"ref_gram_matrix_{prec}")
            fn.argtypes = [_sz, _sz, _p, _sz, _p, _sz, fl, _p, _sz]
            fn.restype = C.c_int
            fn = getattr(L, f"ref_virtual_vis_{prec}")
            fn.argtypes = [fl, _sz, _sz, _p, _p, _sz, _p]
            fn.restype = C.c_int
            fn = getattr(L, f"ref_nuft_sum_{prec}")
            fn.argtypes = [fl, _sz, _p, _p, _p, _p, _sz, _p, _p, _p, _p, C.c_int]
            fn.restype = C.c_int
            fn = getattr(L, f"ref_partition_grid_{prec}")
            fn.argtypes = [_p, _sz, _p, _p, _p, _p, _p, _p]
            fn.restype = C.c_int
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_get_threads.restype = C.c_int
        _lib = L
    return _lib


def _types(dtype):
    if np.dtype(dtype) == np.float32:
        return "f32", np.float32, np.complex64, C.c_float
    return "f64", np.float64, np.complex128, C.c_double


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def set_threads(n: int) -> None:
    lib().ref_set_threads(int(n))


def _check(rc, what):
    if rc != 0:
        raise RuntimeError(f"reference {what} failed with BippError {rc}")


def eigh_gram(wl, s, w, xyz, dtype=np.float64):
    """bipp::eigh_gram (src/eigensolver.cpp:129-225). Returns (v, d, nReduced, scale)."""
    prec, rt, ct, fl = _types(dtype)
    s = np.asfortranarray(s, dtype=ct)
    w = np.asfortranarray(w, dtype=ct)
    xyz = np.asfortranarray(xyz, dtype=rt)
    nA, nB = w.shape
    d = np.zeros(nB, dtype=rt)
    v = np.zeros((nA, nB), dtype=ct, order="F")
    nred = _sz(0)
    scale = fl(0)
    rc = getattr(lib(), f"ref_eigh_gram_{prec}")(
        rt(wl), nA, nB, _ptr(s), nB, _ptr(w), nA, _ptr(xyz), nA, _ptr(d), _ptr(v), nA,
        C.byref(nred), C.byref(scale))
    _check(rc, "eigh_gram")
    return v, d, nred.value, scale.value


def eigh(wl, s, w, dtype=np.float64):
    """bipp::eigh (src/eigensolver.cpp:40-127). Returns (v, d, nReduced, scale)."""
    prec, rt, ct, fl = _types(dtype)
    s = np.asfortranarray(s, dtype=ct)
    w = np.asfortranarray(w, dtype=ct)
    nA, nB = w.shape
    d = np.zeros(nB, dtype=rt)
    v = np.zeros((nA, nB), dtype=ct, order="F")
    nred = _sz(0)
    scale = fl(0)
    rc = getattr(lib(), f"ref_eigh_{prec}")(
        rt(wl), nA, nB, _ptr(s), nB, _ptr(w), nA, _ptr(d), _ptr(v), nA,
        C.byref(nred), C.byref(scale))
    _check(rc, "eigh")
    return v, d, nred.value, scale.value


def gram_matrix(w, xyz, wl, dtype=np.float64):
    """bipp::host::gram_matrix (src/host/gram_matrix.cpp:29-64)."""
    prec, rt, ct, fl = _types(dtype)
    w = np.asfortranarray(w, dtype=ct)
    xyz = np.asfortranarray(xyz, dtype=rt)
    nA, nB = w.shape
    g = np.zeros((nB, nB), dtype=ct, order="F")
    rc = getattr(lib(), f"ref_gram_matrix_{prec}")(nA, nB, _ptr(w), nA, _ptr(xyz), nA, rt(wl), _ptr(g), nB)
    _check(rc, "gram_matrix")
    return g


def virtual_vis(scale, d, v, dtype=np.float64):
    """bipp::host::virtual_vis (src/host/virtual_vis.cpp:19-73); returns VV as a
    column-major nAntenna x nAntenna matrix."""
    prec, rt, ct, fl = _types(dtype)
    v = np.asfortranarray(v, dtype=ct)
    d = np.ascontiguousarray(d, dtype=rt)
    nA, nB = v.shape
    vv = np.zeros(nA * nA, dtype=ct)
    rc = getattr(lib(), f"ref_virtual_vis_{prec}")(rt(scale), nA, nB, _ptr(d), _ptr(v), nA, _ptr(vv))
    _check(rc, "virtual_vis")
    return vv.reshape((nA, nA), order="F")


def nuft_sum(alpha, values, u, v, w, x, y, z, out=None, dtype=np.float64, threads=None):
    """bipp::host::nuft_sum (src/host/kernels/nuft_sum.cpp:9-31): out[p] += Re sum_k
    values_k exp(i alpha (x_p u_k + y_p v_k + z_p w_k))."""
    prec, rt, ct, fl = _types(dtype)
    values = np.ascontiguousarray(values, dtype=ct)
    u, v, w = (np.ascontiguousarray(a, dtype=rt) for a in (u, v, w))
    x, y, z = (np.ascontiguousarray(a, dtype=rt) for a in (x, y, z))
    if out is None:
        out = np.zeros(x.shape[0], dtype=rt)
    nthreads = threads if threads is not None else (os.cpu_count() or 1)
    rc = getattr(lib(), f"ref_nuft_sum_{prec}")(
        rt(alpha), values.shape[0], _ptr(values), _ptr(u), _ptr(v), _ptr(w), x.shape[0],
        _ptr(x), _ptr(y), _ptr(z), _ptr(out), int(nthreads))
    _check(rc, "nuft_sum")
    return out


def partition_grid(dims, x, y, z, dtype=np.float64):
    """bipp::host::DomainPartition::grid (src/host/domain_partition.hpp:35-101).
    Returns (permut, group_begin, group_size); permut[i] is the sorted position of
    point i."""
    prec, rt, ct, fl = _types(dtype)
    x, y, z = (np.ascontiguousarray(a, dtype=rt) for a in (x, y, z))
    n = x.shape[0]
    dims = np.ascontiguousarray(dims, dtype=np.uint64)
    ng = int(np.prod(dims))
    permut = np.zeros(n, dtype=np.uint64)
    gb = np.zeros(max(ng, 1), dtype=np.uint64)
    gs = np.zeros(max(ng, 1), dtype=np.uint64)
    rc = getattr(lib(), f"ref_partition_grid_{prec}")(_ptr(dims), n, _ptr(x), _ptr(y), _ptr(z),
                                                      _ptr(permut), _ptr(gb), _ptr(gs))
    _check(rc, "partition_grid")
    if ng <= 1:
        # DomainPartition::none: a single group, identity order
        return np.arange(n, dtype=np.uint64), np.array([0], np.uint64), np.array([n], np.uint64)
    return permut, gb, gs
