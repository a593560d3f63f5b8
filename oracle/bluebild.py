"""Test infrastructure only: numpy/scipy restatement of the reference's Bluebild path.

This is the CPU oracle that the CUDA path is checked against. It restates, in
FP64 (or the requested precision), what the reference computes; every function
cites the reference file:line it follows (paths relative to the reference
project). It is pinned against the reference's own code compiled by
``oracle/Makefile`` (see ``oracle/ref.py``) and against the golden fixtures in
``tests/golden/``. Only tests, ``__graft_entry__.smoke`` and the CPU-baseline leg
of ``bench.py`` may import it; the product never does.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

TWO_PI = 2.0 * 3.14159265358979323846


class EigensolverError(RuntimeError):
    """The reference's EigensolverError (include/bipp/exceptions.hpp), raised when its LAPACK
    call returns info != 0 (src/host/lapack_api.hpp:88, 109, 133, 157)."""


def _check_reduced(s_red, g=None):
    """The reduced lower triangle of S (and G) must be finite: the reference hands it to
    LAPACK ?heev/?hegv, which reports a NaN/Inf entry as info != 0 (observed with the
    compiled reference sources), raised as EigensolverError."""
    if not np.isfinite(np.tril(s_red)).all() or (g is not None and not np.isfinite(g).all()):
        raise EigensolverError("non-finite entry in the reduced matrix")


# --- flagging + compaction -------------------------------------------------------

def flag_nonzero_gram(s, eps):
    """Rows/cols kept by eigh_gram: |s_ij|^2 > eps in the lower triangle, and
    nVis = count of such entries (diagonal once, off-diagonal twice).
    src/eigensolver.cpp:148-166. |s|^2 is std::norm's re*re + im*im in the precision
    of s (pass s in the working precision for the reference's exact threshold)."""
    s = np.asarray(s)
    low = np.tril(s.real * s.real + s.imag * s.imag > s.real.dtype.type(eps))
    flags = low.any(axis=0) | low.any(axis=1)
    diag = np.diag(low).sum()
    nvis = int(diag + 2 * (low.sum() - diag))
    return np.nonzero(flags)[0], nvis


def flag_nonzero_std(s, eps):
    """Flag test of bipp::eigh: |Re| >= eps or |Im| >= eps (src/eigensolver.cpp:57-76)."""
    s = np.asarray(s)
    e = s.real.dtype.type(eps)
    low = np.tril((np.abs(s.real) >= e) | (np.abs(s.imag) >= e))
    flags = low.any(axis=0) | low.any(axis=1)
    diag = np.diag(low).sum()
    nvis = int(diag + 2 * (low.sum() - diag))
    return np.nonzero(flags)[0], nvis


# --- Gram matrix -------------------------------------------------------------------

def gram_matrix(w, xyz, wl):
    """G = W^H sinc(2|p_i - p_j| / wl) W with sinc(x) = sin(pi x)/(pi x), sinc(0) = 1.
    src/host/gram_matrix.cpp:23-61."""
    xyz = np.asarray(xyz, dtype=np.float64)
    diff = xyz[:, None, :] - xyz[None, :, :]
    dist = np.sqrt((diff ** 2).sum(-1))
    g = np.sinc(2.0 * dist / wl)  # numpy sinc is sin(pi x)/(pi x)
    w = np.asarray(w)
    return w.conj().T @ g @ w


# --- eigensolvers ------------------------------------------------------------------

def eigh_gram(wl, s, w, xyz, dtype=np.float64):
    """Generalized eigenproblem S x = d G x after dropping zero rows/cols of S.
    Returns (v, d, nReduced, scale) with d ascending zero-padded to nBeam,
    v = W_red X zero-padded to nBeam columns, scale = 1/nVis.
    src/eigensolver.cpp:129-225 (LAPACK ?hegv itype 1, src/host/lapack_api.hpp:112-158)."""
    rt = np.dtype(dtype)
    ct = np.complex64 if rt == np.float32 else np.complex128
    eps = float(np.finfo(rt).eps)
    idx, nvis = flag_nonzero_gram(np.asarray(s, dtype=ct), eps)
    if len(idx) == 0:  # LAPACK rejects the 0 x 0 problem's leading dimension 0
        raise EigensolverError("every row and column of S is flagged")
    s = np.asarray(s, dtype=np.complex128)
    w = np.asarray(w, dtype=np.complex128)
    n_ant, n_beam = w.shape
    nred = len(idx)
    d = np.zeros(n_beam, dtype=rt)
    v = np.zeros((n_ant, n_beam), dtype=ct)
    if nred:
        s_red = s[np.ix_(idx, idx)]
        s_red = np.tril(s_red) + np.tril(s_red, -1).conj().T  # lower half is used
        w_red = w[:, idx]
        g = gram_matrix(w_red, xyz, wl)
        _check_reduced(s_red, g)
        try:
            dd, x = sla.eigh(s_red, g)
        except np.linalg.LinAlgError as e:  # G not positive definite: ?hegv info > n
            raise EigensolverError(str(e)) from e
        d[:nred] = dd
        v[:, :nred] = w_red @ x
    scale = 1.0 / nvis if nvis else 0.0
    return v, d, nred, scale


def eigh(wl, s, w, dtype=np.float64):
    """Standard Hermitian eigenproblem after flagging (src/eigensolver.cpp:40-127)."""
    rt = np.dtype(dtype)
    ct = np.complex64 if rt == np.float32 else np.complex128
    eps = float(np.finfo(rt).eps)
    idx, nvis = flag_nonzero_std(np.asarray(s, dtype=ct), eps)
    if len(idx) == 0:  # LAPACK rejects the 0 x 0 problem's leading dimension 0
        raise EigensolverError("every row and column of S is flagged")
    s = np.asarray(s, dtype=np.complex128)
    w = np.asarray(w, dtype=np.complex128)
    n_ant, n_beam = w.shape
    nred = len(idx)
    d = np.zeros(n_beam, dtype=rt)
    v = np.zeros((n_ant, n_beam), dtype=ct)
    if nred:
        s_red = s[np.ix_(idx, idx)]
        _check_reduced(s_red)
        s_red = np.tril(s_red) + np.tril(s_red, -1).conj().T
        dd, x = np.linalg.eigh(s_red)
        d[:nred] = dd
        v[:, :nred] = w[:, idx] @ x
    scale = 1.0 / nvis if nvis else 0.0
    return v, d, nred, scale


# --- virtual visibilities ------------------------------------------------------------

def virtual_vis(scale, d_level, v):
    """VV = V_k diag(scale d_k) V_k^H over the non-zero entries of d_level, as an
    nAnt x nAnt matrix (column-major index i + j nAnt). src/host/virtual_vis.cpp:19-73."""
    d_level = np.asarray(d_level)
    v = np.asarray(v)
    keep = d_level != 0
    if not keep.any():
        return np.zeros((v.shape[0], v.shape[0]), dtype=np.complex128)
    vk = v[:, keep].astype(np.complex128)
    return (vk * (scale * d_level[keep].astype(np.float64))) @ vk.conj().T


# --- energy levels -------------------------------------------------------------------

def centroid_to_intervals(centroid=None, d_min=0.0, d_max=float(np.finfo("f").max)):
    """python/bipp/parameter_estimator.py:18-52."""
    if centroid is None or centroid.size <= 1:
        return np.array([[d_min, d_max]])
    intervals = np.empty((centroid.size, 2))
    sorted_idx = np.argsort(centroid)
    sorted_centroid = centroid[sorted_idx]
    for i in range(centroid.size):
        idx = sorted_idx[i]
        intervals[i, 0] = d_min if idx == 0 else (sorted_centroid[idx] + sorted_centroid[idx - 1]) / 2
        intervals[i, 1] = d_max if idx == centroid.size - 1 else (sorted_centroid[idx] + sorted_centroid[idx + 1]) / 2
    return intervals


def infer_intervals(n_level, sigma, cluster_func, d_min, d_max, d_all):
    """k-means level intervals, seed 42. python/bipp/parameter_estimator.py:55-105."""
    import sklearn.cluster as skcl

    if cluster_func == "log" and d_min < 0:
        raise ValueError(f'Cluster function "log" requires non-negative minimum eigenvalue restriction. Got {d_min}')
    d_all = np.array(d_all).flatten()
    d_all = d_all[d_all != 0.0]
    d_all = d_all[d_all >= d_min]
    d_all = d_all[d_all <= d_max]
    if 0 <= sigma < 1:
        n_remove = int((1 - sigma) * d_all.shape[0])
        if n_remove <= d_all.shape[0]:
            d_all = np.sort(d_all)[0:-n_remove]
    d_all = d_all.reshape(-1, 1)
    if cluster_func == "log":
        km = skcl.KMeans(n_clusters=n_level, random_state=42).fit(np.log(d_all))
        centroid = np.sort(np.exp(km.cluster_centers_)[:, 0])[::-1]
    elif cluster_func == "none":
        km = skcl.KMeans(n_clusters=n_level, random_state=42).fit(d_all)
        centroid = np.sort(km.cluster_centers_[:, 0])[::-1]
    else:
        raise ValueError(cluster_func)
    return centroid_to_intervals(centroid, d_min, d_max)


def apply_filter(name, d):
    """python/bipp/filter.py:7-26."""
    d = np.array(d, dtype=np.float64, copy=True)
    if name == "lsq":
        return d
    if name == "std":
        return np.sign(d)
    if name in ("sqrt", "inv_sqrt"):
        sign = np.sign(d)
        d = sign * np.sqrt(sign * d)
        if name == "inv_sqrt":
            nz = d != 0
            d[nz] = 1.0 / d[nz]
        return d
    if name == "inv":
        nz = d != 0
        d[nz] = 1.0 / d[nz]
        return d
    raise ValueError(name)


def level_eigenvalues(d, lo, hi, filt="lsq"):
    """d_level = filter(d * [lo <= d <= hi]) (python/bipp/filter.py:45-47)."""
    d = np.asarray(d, dtype=np.float64)
    return apply_filter(filt, d * ((d >= lo) & (d <= hi)))


# --- direct NUFT sum -------------------------------------------------------------------

def nuft_sum(alpha, values, u, v, w, x, y, z, chunk=2048):
    """out[p] = sum_k Re(values_k exp(i alpha (x_p u_k + y_p v_k + z_p w_k))), FP64.
    src/host/kernels/nuft_sum.cpp:9-31."""
    values = np.asarray(values, dtype=np.complex128)
    u, v, w = (np.asarray(a, dtype=np.float64) for a in (u, v, w))
    x, y, z = (np.asarray(a, dtype=np.float64) for a in (x, y, z))
    out = np.zeros(x.shape[0])
    for b in range(0, x.shape[0], chunk):
        ph = alpha * (np.outer(x[b:b + chunk], u) + np.outer(y[b:b + chunk], v) + np.outer(z[b:b + chunk], w))
        out[b:b + chunk] = (np.cos(ph) @ values.real) - (np.sin(ph) @ values.imag)
    return out


# --- domain partition ----------------------------------------------------------------

def partition_grid(dims, x, y, z, dtype=np.float64):
    """Bucket permutation of points into a regular grid of groups.
    src/host/domain_partition.hpp:35-101. Returns (permut, begin, size)."""
    rt = np.dtype(dtype)
    coords = [np.asarray(c, dtype=rt) for c in (x, y, z)]
    n = coords[0].shape[0]
    dims = [int(d) for d in dims]
    ng = int(np.prod(dims))
    if ng <= 1:
        return np.arange(n, dtype=np.uint64), np.array([0], np.uint64), np.array([n], np.uint64)
    if n == 0:
        return np.zeros(0, np.uint64), np.zeros(ng, np.uint64), np.zeros(ng, np.uint64)
    gidx = np.zeros(n, dtype=np.int64)
    for dim in (2, 1, 0):
        c = coords[dim]
        cmin, cmax = c.min(), c.max()
        if not cmax > cmin:
            # degenerate extent: the reference's spacing is dims / 0 = inf, inf * 0 = NaN,
            # and its NaN -> size_t conversion (x86-64) clamps to the last cell
            gidx = gidx * dims[dim] + (dims[dim] - 1)
            continue
        inv = rt.type(dims[dim]) / rt.type(cmax - cmin)
        cell = (inv * (c - cmin)).astype(rt)
        # float -> size_t truncation, then clamp to [0, dims-1]
        cell = np.minimum(np.floor(cell).astype(np.int64), dims[dim] - 1)
        cell = np.maximum(cell, 0)
        gidx = gidx * dims[dim] + cell
    size = np.bincount(gidx, minlength=ng).astype(np.uint64)
    begin = np.concatenate([[0], np.cumsum(size)[:-1]]).astype(np.uint64)
    order = np.argsort(gidx, kind="stable")
    permut = np.empty(n, dtype=np.uint64)
    permut[order] = np.arange(n, dtype=np.uint64)
    return permut, begin, size


# --- synthesis ---------------------------------------------------------------------------

def image_synthesis(steps, intervals, lmn, filt="lsq", normalize=True, pixel_idx=None):
    """FP64 image oracle: per step, VV per level (virtual_vis), uvw scaled by 2 pi/wl
    (src/nufft_synthesis.cpp:149-155), direct sum over all nAnt^2 baselines
    (src/host/kernels/nuft_sum.cpp:9-31), real part accumulated
    (src/host/nufft.hpp:208-213), normalised by 1/nSamples
    (src/image_synthesis.cpp:336-347).

    steps: iterable of dicts with keys uvw (nAnt^2 x 3, float32), v (nAnt x nBeam),
    d (nBeam), scale, wl. intervals: (L, 2). lmn: (P, 3). Returns (P_sel, L)."""
    lmn = np.asarray(lmn, dtype=np.float64)
    if pixel_idx is not None:
        lmn = lmn[pixel_idx]
    intervals = np.asarray(intervals, dtype=np.float64)
    n_lvl = intervals.shape[0]
    img = np.zeros((lmn.shape[0], n_lvl))
    n = 0
    for st in steps:
        n += 1
        uvw = np.asarray(st["uvw"], dtype=np.float32).astype(np.float64)
        uvw = uvw * (TWO_PI / float(st["wl"]))
        for lv in range(n_lvl):
            dl = level_eigenvalues(st["d"], intervals[lv, 0], intervals[lv, 1], filt)
            vv = virtual_vis(float(st["scale"]), dl, st["v"])
            vals = vv.reshape(-1, order="F")
            img[:, lv] += nuft_sum(1.0, vals, uvw[:, 0], uvw[:, 1], uvw[:, 2],
                                   lmn[:, 0], lmn[:, 1], lmn[:, 2])
    if normalize and n:
        img /= n
    return img
