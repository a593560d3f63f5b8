"""FP64 check of the batched pipeline on the GPU, for large batches.

The FP32 pipeline (the form the benchmark times) images a batch of time steps; the
same steps are then imaged in FP64 by this library's own FP64 pieces, each pinned to
the reference's CPU code by the parity tests:

- eigenpairs: ``bipp_eigh_gram_batched_d`` (the reference's eigh_gram<double>, i.e.
  zhegv after flagging, src/eigensolver.cpp:129-225);
- virtual visibilities: VV_l = V diag(scale * d * [lo_l <= d <= hi_l]) V^H in FP64
  (src/host/virtual_vis.cpp:19-73, the level mask of python/bipp/filter.py:45-47);
- image: the direct sum out[p] = sum_k Re(VV_k exp(i (x_p u_k + y_p v_k + z_p w_k)))
  over all N^2 baselines (src/host/kernels/nuft_sum.cpp:9-31), with the phase formed and
  reduced and its sine and cosine taken in FP64 (``bipp_nuft_sum_multi_device``, VV
  rounded to complex64, a relative perturbation of 6e-8), on a random pixel subset;
- normalisation 1/nSteps (src/image_synthesis.cpp:152-163).

Returned: the relative L2 error of the pipeline's level images at those pixels, and the
eigenvalue errors of the pipeline's eigenvalues inside the level range, per eigenvalue
(|d - d64| / |d64|) and normwise (max |d - d64| / max |d64|).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check


def _lattice(lmn, n):
    l = lmn[:, 0].reshape(n, n)
    m = lmn[:, 1].reshape(n, n)
    return (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])


def fp64_level_images(ctx, s_logical, xyz, wl, basis, intervals, lmn_pix, chunk=32):
    """FP64 level images [L, P] (normalised by the number of steps) and eigenvalues
    [B, N] of the steps s_logical [B, N, N] (complex, S[i, j]), xyz [B, N, 3], wl [B]."""
    import torch

    from .api import eigh_gram_batched

    B, N = s_logical.shape[0], s_logical.shape[1]
    L = intervals.shape[0]
    dev = torch.device("cuda", ctx.device if ctx.device is not None else torch.cuda.current_device())
    px = [torch.from_numpy(np.ascontiguousarray(lmn_pix[:, c], dtype=np.float64)).to(dev) for c in range(3)]
    P = lmn_pix.shape[0]
    out = torch.zeros((L, P), dtype=torch.float64, device=dev)
    vals = torch.empty((L, N * N), dtype=torch.complex64, device=dev)
    d_all = np.zeros((B, N))
    for b0 in range(0, B, chunk):
        nb = min(chunk, B - b0)
        v, d, nred, scale = eigh_gram_batched(wl[b0:b0 + nb], s_logical[b0:b0 + nb], xyz[b0:b0 + nb], ctx=ctx,
                                              precision="double")
        d_all[b0:b0 + nb] = d
        for k in range(nb):
            vk = torch.from_numpy(np.ascontiguousarray(v[k])).to(dev)        # [N, N], column c = eigenvector c
            dk = torch.from_numpy(d[k]).to(dev)
            for lv in range(L):
                lo, hi = float(intervals[lv, 0]), float(intervals[lv, 1])
                f = dk * ((dk >= lo) & (dk <= hi)).to(torch.float64) * float(scale[k])
                vv = (vk * f) @ vk.conj().T                                  # VV[i, j]
                vals[lv] = vv.T.reshape(-1).to(torch.complex64)              # index i + j N
            au = np.asarray(xyz[b0 + k], dtype=np.float64) @ basis
            bl = (au[:, None, :] - au[None, :, :]).transpose(1, 0, 2).reshape(-1, 3) * (2.0 * math.pi / wl[b0 + k])
            bt = torch.from_numpy(np.ascontiguousarray(bl.T)).to(dev)        # [3, N^2]: u, v, w
            # torch wrote vals and bt on its stream; the library call runs on the
            # context's stream (and synchronises it before returning)
            torch.cuda.current_stream(dev).synchronize()
            check(ctx._lib.bipp_nuft_sum_multi_device(
                ctx.handle, C.c_double(1.0), N * N, L, C.c_void_p(vals.data_ptr()), N * N,
                C.c_void_p(bt[0].data_ptr()), C.c_void_p(bt[1].data_ptr()), C.c_void_p(bt[2].data_ptr()), P,
                C.c_void_p(px[0].data_ptr()), C.c_void_p(px[1].data_ptr()), C.c_void_p(px[2].data_ptr()),
                C.c_void_p(out.data_ptr()), P, 1))
    return (out / B).cpu().numpy(), d_all


def eigenvalue_errors(d_pipe, d64, intervals):
    """Errors of the pipeline's eigenvalues inside the level range [min lo, max hi]
    against the FP64 ones: max per-eigenvalue relative error |d - d64| / |d64| over all of
    them and over those with |d64| >= 1e-2 max|d64| of their step, the max normwise error
    |d - d64| / max|d64|, and the number compared. An FP32 solver's eigenvalue error is of
    the order of eps32 times the norm, so the relative error of the smallest eigenvalues
    is larger by max|d| / |d| (the reference's own FP32 path, chegv, shows the same).
    Eigenvalues within 1e-6 max|d| of a range edge are left out (FP32 may place them on
    the other side)."""
    lo, hi = float(intervals[:, 0].min()), float(intervals[:, 1].max())
    per, large, norm, n = 0.0, 0.0, 0.0, 0
    for b in range(d64.shape[0]):
        ref = d64[b]
        scale = np.abs(ref).max()
        if scale == 0:
            continue
        edge = 1e-6 * scale
        sel = (ref >= lo + edge) & (ref <= hi - edge)
        if not sel.any():
            continue
        diff = np.abs(d_pipe[b][sel] - ref[sel])
        rel = diff / np.abs(ref[sel])
        per = max(per, float(rel.max()))
        big = np.abs(ref[sel]) >= 1e-2 * scale
        if big.any():
            large = max(large, float(rel[big].max()))
        norm = max(norm, float(diff.max() / scale))
        n += int(sel.sum())
    return {"eig_rel_err_max": per, "eig_rel_err_max_above_1e-2": large, "eig_rel_err_normwise": norm,
            "eigenvalues_compared": n}


def check_batch(ctx, S_cm, xyz, wl, obs, image_size, intervals, tolerance, n_pix=512, seed=33, chunk_steps=None,
                filter="lsq", vv_precision="tf32x3"):
    """Image the steps of S_cm (torch device tensor [B, N, N], each step's S in
    column-major order, complex64), xyz (torch [B, N, 3] float64), wl (torch [B] float64)
    with the FP32 pipeline and with the FP64 pieces; returns a dict of errors and the
    pipeline's NUFFT statistics."""
    import torch

    from .api import Pipeline

    if filter != "lsq":
        raise ValueError("the FP64 check implements the 'lsq' filter")
    B, N = S_cm.shape[0], S_cm.shape[1]
    n = image_size
    pl = Pipeline(ctx, N, intervals, _lattice(obs.lmn, n), obs.lmn[:, 2], obs.basis, tolerance=tolerance,
                  chunk_steps=chunk_steps or B, max_steps=B, vv_precision=vv_precision)
    pl.process_device(B, S_cm.data_ptr(), xyz.data_ptr(), wl.data_ptr())
    img = pl.images()
    stats = pl.nufft_stats()
    d_pipe, _ = pl.last_eigenvalues(B)
    pl.close()
    torch.cuda.synchronize()
    pix = np.random.default_rng(seed).choice(obs.lmn.shape[0], n_pix, replace=False)
    s_log = S_cm.transpose(1, 2).cpu().numpy().astype(np.complex128)
    ref, d64 = fp64_level_images(ctx, s_log, xyz.cpu().numpy(), wl.cpu().numpy(), obs.basis, intervals,
                                 obs.lmn[pix])
    got = img[:, pix].astype(np.float64)
    err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
    out = {"image_rel_l2": err}
    out.update(eigenvalue_errors(d_pipe, d64, np.asarray(intervals)))
    out.update({"steps": int(B), "pixels": int(n_pix), "split_tiles": stats["split_tiles"], "slabs": stats["slabs"],
                "points": stats["points"]})
    return out
