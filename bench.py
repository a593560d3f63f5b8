#!/usr/bin/env python
"""Bluebild imaging throughput: time-steps/s at 512 antennas and a 1024^2 image.

Workload (one bench step = one batch): 2048 time steps of a 512-antenna log-radial
array (35 km), 380-512 antennas kept per step, 200-source sky, 4 energy levels,
1024 x 1024 pixel lattice over 16 deg, NUFFT tolerance 1e-5; per time step: flagging,
Gram, generalized eigensolve, level binning, virtual visibilities, NUFFT synthesis.
Seeded synthetic inputs (the reference's datasets are not available); inputs (4.3 GB of
visibilities per batch) are larger than L2, so no extra flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

--impl reference times the reference's own CPU code (oracle/_ref, compiled from the
reference sources) on the host cores, on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "time-steps/s at 512 antennas, 1024^2 px (4 levels, NUFFT eps 1e-5)"
METRIC_C5 = "time-steps/s at 1024 antennas, 8 channels, 2048^2 px (8 levels, NUFFT eps 1e-5)"
UNIT = "time-steps/s"


def metric_of(args):
    return METRIC_C5 if args.workload == "c5" else METRIC


def workload_text(args):
    if args.workload == "c5":
        return (f"c5: {args.antennas} antennas log-radial 50 km, 25% flagged/step, 8 channels 1.5-3 m, 500 sources, "
                f"8 levels, {args.image}^2 px over 16 deg, eps 1e-5; {args.time_steps} of 4096 time steps")
    return (f"c2: {args.antennas} antennas log-radial 35 km, 380-512 kept/step, 200 sources, 4 levels, "
            f"{args.image}^2 px over 16 deg, eps 1e-5")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c2", "c5", "c4", "c2-api"],
                    help="c2: 512 antennas, 2048 steps, 1024^2 px, 4 levels (the headline); c5: 1024 antennas, "
                         "8 frequency channels, 2048^2 px, 8 levels (bounded to --time-steps time steps); c4: the "
                         "learned rank predictor study (256 antennas; eigensolver only)")
    ap.add_argument("--time-steps", type=int, default=None)
    ap.add_argument("--antennas", type=int, default=None)
    ap.add_argument("--image", type=int, default=None)
    ap.add_argument("--mode", default="batched", choices=["batched", "plain"])
    ap.add_argument("--chunk-steps", type=int, default=None, help="entries per eigensolver/VV chunk")
    ap.add_argument("--vv-precision", default="tf32x3", choices=["tf32x3", "bf16x3", "fp32", "fp64"],
                    help="arithmetic of the virtual-visibility products of the batched form")
    ap.add_argument("--e2e-steps", type=int, default=8)
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default launch shapes instead of tuning them on the batch first")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--stages", action="store_true", help="report per-stage device times")
    ap.add_argument("--check-steps", type=int, default=256,
                    help="entries of the FP64 image/eigenvalue check (spread over the batch); 0 skips it")
    ap.add_argument("--check-pixels", type=int, default=512)
    ap.add_argument("--plain-steps", type=int, default=16,
                    help="time steps of the plain-GPU comparison (one NUFFT per step and level); 0 skips it")
    a = ap.parse_args()
    dflt = {"c2": dict(time_steps=2048, antennas=512, image=1024, chunk_steps=2048),
            "c5": dict(time_steps=128, antennas=1024, image=2048, chunk_steps=592),
            "c4": dict(time_steps=10000, antennas=256, image=256, chunk_steps=2000),
            "c2-api": dict(time_steps=128, antennas=512, image=1024, chunk_steps=128)}[a.workload]
    for k, v in dflt.items():
        if getattr(a, k) is None:
            setattr(a, k, v)
    return a


def workload_config(args, seed_offset=0):
    from bipp_b200 import simulate as sim

    if args.workload == "c5":
        return sim.config_c5(n_antenna=args.antennas, image_size=args.image, n_steps=args.time_steps,
                             keep=(args.antennas * 3 // 4, args.antennas * 3 // 4), seed=5 + seed_offset)
    return sim.config_c2(n_antenna=args.antennas, image_size=args.image, n_steps=args.time_steps, seed=2 + seed_offset)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_inputs(cfg, rank, device):
    """Seeded inputs on the GPU, one entry per (time step, frequency channel), entry
    t * n_channels + c: S^T (column-major S), xyz, wl. Ranks differ only in the noise."""
    import torch

    from bipp_b200 import simulate as sim

    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    T, N, C = cfg.n_steps, cfg.n_antenna, cfg.n_channels
    wls = cfg.wavelengths()
    S = torch.empty((T * C, N, N), dtype=torch.complex64, device=device)
    xyz = torch.empty((T * C, N, 3), dtype=torch.float64, device=device)
    wl = torch.empty((T * C,), dtype=torch.float64, device=device)
    chunk = 64 if N <= 512 else 16
    for s0 in range(0, T, chunk):
        steps = list(range(s0, min(T, s0 + chunk)))
        for c in range(C):
            s, x = sim.visibilities(obs, steps, device=device, dtype=torch.complex64, masks=masks, wl=float(wls[c]),
                                    noise_key=c + 64 * rank)
            S[s0 * C + c:(s0 + len(steps)) * C:C] = s.transpose(1, 2)
            xyz[s0 * C + c:(s0 + len(steps)) * C:C] = x
            wl[s0 * C + c:(s0 + len(steps)) * C:C] = float(wls[c])
    torch.cuda.synchronize()
    return obs, S, xyz, wl


def lower_block_bytes(n, t, cols=64):
    """Bytes of visibilities a host-input pipeline call copies: the lower triangle of each
    n x n complex64 matrix in blocks of `cols` columns, from each block's diagonal down."""
    return t * 8 * sum((n - c0) * min(cols, n - c0) for c0 in range(0, n, cols))


def lattice_of(obs, n):
    l = obs.lmn[:, 0].reshape(n, n)
    m = obs.lmn[:, 1].reshape(n, n)
    return (n, n, l[0, 0], m[0, 0], l[1, 0] - l[0, 0], l[0, 1] - l[0, 0], m[1, 0] - m[0, 0], m[0, 1] - m[0, 0])


def calibrate_levels(ctx, cfg, S, xyz, wl, n_cal=64):
    """Energy levels: k-means (log) over positive eigenvalues of the first n_cal entries
    (python/bipp/parameter_estimator.py:55-105), then frozen."""
    import bipp_b200 as bipp
    from bipp_b200.parameter_estimator import infer_intervals

    n_cal = min(n_cal, S.shape[0])
    s_host = S[:n_cal].transpose(1, 2).cpu().numpy()
    x_host = xyz[:n_cal].cpu().numpy()
    w_host = wl[:n_cal].cpu().numpy().astype(np.float32)
    _, d, nred, _ = bipp.eigh_gram_batched(w_host, s_host, x_host, ctx=ctx)
    return infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, d)


def share_levels(intervals, device):
    """Rank 0's energy-level intervals on every rank (a broadcast in the default process
    group), so that the level images of all ranks add up."""
    import torch
    import torch.distributed as dist

    iv = torch.from_numpy(np.ascontiguousarray(intervals, dtype=np.float64)).to(device)
    dist.broadcast(iv, src=0)
    return iv.cpu().numpy()


def cpu_reference_sample(cfg, S, xyz, intervals, n_eig_steps=5, n_pix=2048, threads=None, wl=None, nufft=True,
                         ref_eig_errors=False):
    """The reference's CPU path (compiled reference sources) on a bounded sample.

    Measured in full: eigh_gram<float> + virtual_vis<float> for every level, per entry,
    on n_eig_steps entries; the rate is the median over those entries (time-steps/s, a
    time step holding cfg.n_channels entries). The NUFFT stage has no CPU counterpart here
    (the reference's neonufft is not available): when `nufft` is set, the reference's
    direct sum nuft_sum<double> over all baselines of one entry is timed on n_pix pixels
    and extrapolated to the full image and all levels, reported separately and never
    folded into the rate. Returns (time-steps/s, cores, sample description, extras)."""
    from oracle import ref

    from bipp_b200 import simulate as sim

    threads = threads or os.cpu_count() or 1
    wl = float(cfg.wavelengths()[0]) if wl is None else wl
    ref.set_threads(threads)
    obs = sim.observation(cfg)
    N = cfg.n_antenna
    w = np.eye(N, dtype=np.complex64)
    t_eig, t_vv = [], []
    last = None
    for k in range(n_eig_steps):
        s = S[k].transpose(0, 1).cpu().numpy().T  # logical S
        x = xyz[k].cpu().numpy().astype(np.float32)
        t0 = time.perf_counter()
        v, d, nr, sc = ref.eigh_gram(wl, s, w, x, dtype=np.float32)
        t1 = time.perf_counter()
        vvs = []
        for lo, hi in intervals:
            vvs.append(ref.virtual_vis(sc, d * ((d >= lo) & (d <= hi)), v, dtype=np.float32))
        t2 = time.perf_counter()
        t_eig.append(t1 - t0)
        t_vv.append(t2 - t1)
        last = (vvs, xyz[k].cpu().numpy())
    per_entry = float(np.median(np.add(t_eig, t_vv)))
    # the reference FP32 eigenvalues' own error against its FP64 path (zhegv) on the
    # same entries, beside which the GPU's eigenvalue error is read
    if ref_eig_errors:
        from bipp_b200.verify import eigenvalue_errors

        d32, d64 = [], []
        for k in range(n_eig_steps):
            s = S[k].transpose(0, 1).cpu().numpy().T.astype(np.complex128)
            x = xyz[k].cpu().numpy().astype(np.float32)
            d32.append(ref.eigh_gram(wl, s.astype(np.complex64), w, x, dtype=np.float32)[1])
            d64.append(ref.eigh_gram(wl, s, np.eye(N), x.astype(np.float64), dtype=np.float64)[1])
        ref_err = eigenvalue_errors(np.array(d32, dtype=np.float64), np.array(d64), np.asarray(intervals))
    else:
        ref_err = None
    rate = 1.0 / (per_entry * cfg.n_channels)
    desc = (f"eigh_gram<float>+virtual_vis<float>x{len(intervals)} measured on {n_eig_steps} entries, median "
            f"{per_entry:.3f} s/entry (eigh_gram {np.median(t_eig):.3f}, virtual_vis {np.median(t_vv):.4f}); "
            f"{cfg.n_channels} entries per time step; NUFFT stage not included (neonufft unavailable)")
    extras = {"eig_vv_s_per_entry": per_entry}
    if ref_err:
        extras["reference_fp32_eig_errors"] = ref_err
    if nufft:
        vvs, x = last
        uvw = sim.baseline_uvw(obs, x).astype(np.float64) * (2 * math.pi / wl)
        rng = np.random.default_rng(0)
        pix = rng.choice(obs.lmn.shape[0], n_pix, replace=False)
        lmn = obs.lmn[pix]
        vals = vvs[0].reshape(-1, order="F").astype(np.complex128)
        t0 = time.perf_counter()
        ref.nuft_sum(1.0, vals, uvw[:, 0], uvw[:, 1], uvw[:, 2], lmn[:, 0], lmn[:, 1], lmn[:, 2], threads=threads)
        t_pix = time.perf_counter() - t0
        t_nuft = t_pix * (obs.lmn.shape[0] / n_pix) * len(intervals)
        extras["nufft_direct_sum_extrapolated"] = {
            "s_per_entry": round(t_nuft, 1), "kind": "extrapolated",
            "sample": f"nuft_sum<double> over all {N * N} baselines x {n_pix} px measured ({t_pix:.2f} s), scaled to "
                      f"{obs.lmn.shape[0]} px x {len(intervals)} levels; an O(baselines x pixels) direct sum, not "
                      f"the reference's NUFFT"}
    return rate, threads, desc, extras


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "of measured"
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "of fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per algorithmic byte of the
# spreading kernel (FP16 hi/lo operands), measured with ncu over all three spreading
# launches of a 128-step batch of this workload (512 antennas, 1024^2 px, 4 levels, 2 GB
# w-slabs): 4.742e9 DRAM bytes for 5.493e9 algorithmic bytes. The traffic of a full launch is taken to scale with
# the points and cells it processes, as the algorithmic bytes do (tiles without points are
# cleared by their own kernel, so the ratio is below 1).
SPREAD_TRAFFIC_PER_ALG_BYTE = 0.863


def spread_roofline(stats, spread_ms, n_levels):
    """Roofline of the dominant NUFFT kernel, the spreader (one launch per w-slab).

    Algorithmic bytes of one batch: every point read once (3 FP32 coordinates + one
    complex FP32 value per level) and every fine-grid cell written once per level:
    points * (12 + 8 L) + L * cells * 8 (= the grid bytes). Per launch = batch / slabs;
    the launch duration is the spreading kernels' CUDA-event time / slabs."""
    slabs = max(1, stats["slabs"])
    bytes_batch = stats["points"] * (12 + 8 * n_levels) + stats["grid_bytes"]
    per_launch = bytes_batch / slabs
    dur_s = spread_ms / 1000.0 / slabs
    peaks, label = measured_peaks()
    achieved = per_launch / dur_s / 1e9
    flops = stats["points"] * n_levels * 4 * stats["W"] ** 3 / slabs  # real weight x complex value: 4 flops
    ratio = SPREAD_TRAFFIC_PER_ALG_BYTE
    traffic = int(ratio * per_launch) if ratio else None
    return {"kernel": "spread_tc_kernel", "bound": "hbm", "achieved": round(achieved, 2),
            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": round(achieved / peaks["hbm_gbs"], 5),
            "peak_source": label, "traffic": traffic, "algorithmic_bytes_per_launch": int(per_launch),
            "launches_per_step": slabs, "launch_ms": round(dur_s * 1000.0, 3),
            "flops_per_launch": int(flops), "achieved_tflops": round(flops / dur_s / 1e12, 3),
            "note": spread_operands_note() + "; bound by building the dense operands (latency at "
                    "32 warps per SM), the HBM fraction is its floor"}


def spread_operands_note():
    """Which operand form the spreader ran with (the tuning table's spread.operands)."""
    import bipp_b200 as bipp

    mode = bipp.tuning_get("spread.operands")
    return {0: "tcgen05 kind::tf32 spreading, 3xTF32 split, A in shared memory",
            1: "tcgen05 kind::tf32 spreading, 3xTF32 split, A in tensor memory",
            2: "tcgen05 kind::f16 spreading, FP16 hi/lo split (3 MMAs), values scaled per level"}.get(mode, str(mode))


def run_reference(args):
    """--impl reference: the reference's CPU implementation on host cores (rank 0 only)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import torch

    from bipp_b200 import simulate as sim

    args.time_steps = max(8, args.steps + args.warmup)  # one entry per bench step
    cfg = workload_config(args)
    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    wl0 = float(cfg.wavelengths()[0])
    s, x = sim.visibilities(obs, list(range(cfg.n_steps)), dtype=torch.complex64, masks=masks, wl=wl0)
    S = s.transpose(1, 2)
    from bipp_b200.parameter_estimator import infer_intervals
    from oracle import ref

    ref.set_threads(os.cpu_count() or 1)
    d_all = []
    for k in range(2):
        _, d, _, _ = ref.eigh_gram(wl0, s[k].numpy(), np.eye(cfg.n_antenna), x[k].numpy().astype(np.float32),
                                   dtype=np.float32)
        d_all.append(d)
    intervals = infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, np.concatenate(d_all))
    # each bench step: eigh_gram<float> + virtual_vis<float> per level on one entry
    # (measured in full); the NUFFT stage is reported apart (its direct-sum
    # extrapolation), not folded into the value
    vals = []
    for k in range(args.warmup + args.steps):
        v, cores, desc, _ = cpu_reference_sample(cfg, S[k:k + 1], x[k:k + 1], intervals, n_eig_steps=1, wl=wl0,
                                                 nufft=False)
        if k >= args.warmup:
            vals.append(v)
    value = float(np.median(vals))
    _, _, _, extra = cpu_reference_sample(cfg, S[:1], x[:1], intervals, n_eig_steps=1, n_pix=1024, wl=wl0)
    desc = (f"eigh_gram<float>+virtual_vis<float>x{cfg.n_levels} per entry, median of {args.steps} entries "
            f"({1.0 / value:.3f} s per time step); NUFFT stage not included (neonufft unavailable)")
    line = {"impl": "reference", "metric": metric_of(args), "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded observation of the workload's shape)",
            "config": {"workload": workload_text(args), "sample": "one entry (time step x channel) per bench step",
                       "stages_timed": "eigh_gram + virtual_vis (the reference's CPU path for them)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc},
            "nufft_direct_sum_extrapolated": extra.get("nufft_direct_sum_extrapolated"),
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_rank_study(args):
    """--workload c4: the learned rank predictor on the 256-antenna workload. The MLP is
    trained on the GPU on the first 2000 steps (features and labels from the method's own
    full solve); the other steps are solved by the full solve (every eigenpair), the exact
    range above the threshold (Sturm counts) and the predicted partial solve (k + 16,
    fallback to full). Eigensolver device time per mode, fallback rate, count error and
    the partial solve's eigenvalue error against the full solve."""
    import torch

    import bipp_b200 as bipp
    from bipp_b200 import rank
    from bipp_b200 import simulate as sim

    torch.cuda.set_device(0)
    ctx = bipp.Context("GPU", device=0)
    cfg = sim.config_c4(n_steps=args.time_steps, n_antenna=args.antennas)
    obs = sim.observation(cfg)
    n_train = min(2000, args.time_steps // 2)
    r = rank.study(ctx, obs, n_train=n_train, n_eval=args.time_steps - n_train, chunk=args.chunk_steps)
    r.pop("model")
    rates = r["steps_per_s"]
    line = {"metric": "time-steps/s of the eigensolver at 256 antennas (rank-predictor workload)",
            "value": rates["predicted"], "unit": UNIT, "n_gpus": 1, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded per-step skies and noise levels)",
            "config": {"workload": f"c4: {cfg.n_antenna} antennas in a 10 km disc, {args.time_steps} time steps, "
                                   f"5-200 sources and noise 0.001-0.1 per step, threshold 0"},
            "rank_study": r}
    print(json.dumps(line))
    ctx.close()


def run_api_synthesis(args):
    """--workload c2-api: image synthesis through the reference-facing API, the way a
    reference caller images a dataset (bipp::image_synthesis / pybipp image_synthesis over
    a Dataset whose samples hold eigenvectors, eigenvalues, uvw, wl and scale): an
    in-memory dataset of --time-steps steps of the 512-antenna workload (eigenpairs from
    the library's batched eigh_gram), 4 energy-level images of the 1024^2 lattice. Timed:
    the whole call (dataset reads through host callbacks, uvw copies, virtual visibilities
    on the GPU written into the collectors, NUFFT, images back to the host)."""
    import torch

    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    torch.cuda.set_device(0)
    ctx = bipp.Context("GPU", device=0)
    n_steps = args.time_steps
    cfg = sim.config_c2(n_steps=2048)
    obs = sim.observation(cfg)
    masks = sim.keep_masks(cfg)
    steps = list(range(0, 2048, max(1, 2048 // n_steps)))[:n_steps]
    s, x = sim.visibilities(obs, steps, masks=masks)
    s, x = s.numpy(), x.numpy()
    wl = np.full(len(steps), cfg.wl, np.float32)
    v, d, nred, scale = bipp.eigh_gram_batched(wl, s, x, ctx=ctx)
    from bipp_b200.parameter_estimator import infer_intervals

    intervals = infer_intervals(cfg.n_levels, 1.0, "log", 0.0, np.inf, d[:64])
    ds = bipp.InMemoryDataset(cfg.n_antenna, cfg.n_antenna)
    for k in range(len(steps)):
        ds.write(k, cfg.wl, scale[k], v[k], d[k], sim.baseline_uvw(obs, x[k]))
    sel = {f"lvl{l}": {k: d[k] * ((d[k] >= lo) & (d[k] <= hi)) for k in range(len(steps))}
           for l, (lo, hi) in enumerate(intervals)}
    opt = bipp.NufftSynthesisOptions().set_tolerance(cfg.eps).set_normalize_image(True)
    lmn = obs.lmn.astype(np.float32)
    bipp.image_synthesis(ctx, opt, ds, {t: dict(list(m.items())[:2]) for t, m in sel.items()}, lmn)   # warm-up
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        bipp.image_synthesis(ctx, opt, ds, sel, lmn)
        times.append(time.perf_counter() - t0)
    sec = float(np.median(times))
    line = {"metric": "time-steps/s of image synthesis from a dataset (reference API) at 512 antennas, 1024^2 px",
            "value": len(steps) / sec, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "higher_is_better": True,
            "dtype": "f32", "data": "synthetic (seeded observation of the workload's shape; eigenpairs precomputed)",
            "config": {"workload": f"c2-api: {len(steps)} samples of the 512-antenna workload in an in-memory dataset, "
                                   "4 energy-level images, 1024^2 lattice, eps 1e-5",
                       "api": "bipp_b200.image_synthesis -> bipp_image_synthesis (the C++ bipp::image_synthesis "
                              "calls the same entry point)"},
            "s_per_call": sec}
    print(json.dumps(line))
    ctx.close()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "c4":
        run_rank_study(args)
        return
    if args.workload == "c2-api":
        run_api_synthesis(args)
        return
    import torch
    import torch.distributed as dist

    import bipp_b200 as bipp
    from bipp_b200 import simulate as sim

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    ctx = bipp.Context("GPU", device=local)
    # every rank images its own batch of the same observation (array, sky, flags), with
    # its own noise draw
    cfg = workload_config(args)
    obs, S, xyz, wl = make_inputs(cfg, rank, device)
    intervals = calibrate_levels(ctx, cfg, S, xyz, wl)
    if world > 1:
        intervals = share_levels(intervals, device)
    n = cfg.image_size
    pl = bipp.Pipeline(ctx, cfg.n_antenna, intervals, lattice_of(obs, n), obs.lmn[:, 2], obs.basis,
                       tolerance=cfg.eps, chunk_steps=min(args.chunk_steps, S.shape[0]), max_steps=S.shape[0],
                       mode=args.mode, vv_precision=args.vv_precision if args.mode == "batched" else "fp32")
    T = S.shape[0]  # entries: time steps x channels
    S_bytes = S.numel() * 8
    T_steps = cfg.n_steps
    stream = torch.cuda.ExternalStream(ctx.stream(), device=device)

    def one_step():
        pl.process_device(T, S.data_ptr(), xyz.data_ptr(), wl.data_ptr())

    # launch shapes tuned on this batch before the warm-up (the tuned values stay in the
    # process's tuning table for the timed region)
    tuning = None
    if args.autotune and args.mode == "batched":
        tuning = pl.autotune(T, S.data_ptr(), xyz.data_ptr(), wl.data_ptr(), on_device=True, repeats=2)
    for _ in range(args.warmup):
        one_step()
    pl.reset()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n_launch0 = bipp.kernel_launch_count()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            one_step()
        ev1.record(stream)
        torch.cuda.synchronize()
    gpu_launches = bipp.kernel_launch_count() - n_launch0
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    ms_t = torch.tensor([ms], device=device, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = args.steps * T_steps * world / (ms_max / 1000.0)

    # images: one reduction of the level images over ranks per run (SUM, to rank 0)
    img = torch.empty((cfg.n_levels, n * n), dtype=torch.float32, device=device)
    pl.images_device(img.data_ptr(), normalize=False)
    if world > 1:
        dist.reduce(img, dst=0, op=dist.ReduceOp.SUM)

    # per-stage breakdown (separate, untimed pass)
    stages = roof = None
    if args.stages or rank == 0:
        pl.reset()
        pl.stage_times(True)
        one_step()
        st = pl.stage_times(False)
        stages = dict(zip(["eigensolve", "levels_vv", "flags_sort_scatter", "spread", "fft", "wsum", "grid_clear"],
                          [round(float(x), 3) for x in st]))
        kt = pl.kernel_times()
        stages["eig_kernels"] = dict(zip(["prep_gram", "cholesky_fp64", "trinv_fp64", "reduction_gemms", "hetrd",
                                          "tridiag_fp64", "backtransform", "x_gemm"], [round(float(x), 3) for x in kt]))
        roof = spread_roofline(pl.nufft_stats(), float(st[3]), cfg.n_levels)
        # the stages the CPU baseline times in full (eigensolve + levels/virtual
        # visibilities), as a rate of the same unit
        stages["eig_vv_rate"] = {"value": T_steps / ((float(st[0]) + float(st[1])) / 1000.0), "unit": UNIT,
                                 "stages": "eigensolve + levels_vv"}

    # image and eigenvalue error of the timed form against FP64, on a sub-batch spread
    # over the whole batch (every (T / check_steps)-th entry), at random pixels
    parity = None
    if rank == 0 and args.check_steps > 0:
        from bipp_b200 import verify

        stride = max(1, T // args.check_steps)
        sel = torch.arange(0, T, stride, device=device)[:args.check_steps]
        try:
            parity = verify.check_batch(ctx, S[sel].contiguous(), xyz[sel].contiguous(), wl[sel].contiguous(), obs,
                                        n, intervals, cfg.eps, n_pix=args.check_pixels,
                                        chunk_steps=min(args.chunk_steps, len(sel)), vv_precision=args.vv_precision)
            parity["reference"] = ("FP64: bipp_eigh_gram_batched_d + FP64 V diag(d) V^H + direct sum with FP64 "
                                   "phase and trigonometry (the library's FP64 pieces pinned to the compiled "
                                   "reference)")
        except bipp.GPUError as err:
            # a second pipeline beside the benchmark's (larger workloads): reported, not fatal
            parity = {"skipped": str(err)[:200], "hint": "lower --check-steps"}

    # the plain GPU form of the metric on a bounded sample: the same kernels, one step at a
    # time and one NUFFT per step and level (no batching across steps or levels)
    plain = None
    if rank == 0 and args.plain_steps > 0 and args.mode == "batched":
        ns = min(args.plain_steps * cfg.n_channels, T)
        pp = bipp.Pipeline(ctx, cfg.n_antenna, intervals, lattice_of(obs, n), obs.lmn[:, 2], obs.basis,
                           tolerance=cfg.eps, chunk_steps=1, max_steps=ns, mode="plain", vv_precision="fp32")
        pp.process_device(ns, S.data_ptr(), xyz.data_ptr(), wl.data_ptr())  # warm-up
        pp.reset()
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        p0.record(stream)
        pp.process_device(ns, S.data_ptr(), xyz.data_ptr(), wl.data_ptr())
        p1.record(stream)
        torch.cuda.synchronize()
        pv = ns / cfg.n_channels / (p0.elapsed_time(p1) / 1000.0)
        plain = {"value": pv, "unit": UNIT, "sample": f"first {ns} entries (time step x channel) of the batch",
                 "chosen_over_plain": value / pv}
        pp.close()

    # end to end through the public API: pinned host inputs copied in every step,
    # images read back every step
    e2e = None
    if not args.no_e2e:
        S_h = torch.empty(S.shape, dtype=S.dtype, pin_memory=True)
        S_h.copy_(S)
        xyz_h = xyz.cpu().pin_memory()
        wl_h = wl.cpu().pin_memory()
        img_h = torch.empty((cfg.n_levels, n * n), dtype=torch.float32, pin_memory=True)
        del S
        torch.cuda.empty_cache()
        pl.reset()
        pl.process_host_ptr(T, S_h.data_ptr(), xyz_h.data_ptr(), wl_h.data_ptr())  # warm-up
        pl.stage_host_ptr(T, S_h.data_ptr(), xyz_h.data_ptr(), wl_h.data_ptr())
        pl.process_staged()
        torch.cuda.synchronize()
        # every batch is copied in from pinned host memory inside the timed region; batch
        # k + 1 is staged (its copy runs on the library's copy stream) before batch k is
        # processed, so the copies after the first overlap the previous batch's work
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        e0.record(stream)
        pl.stage_host_ptr(T, S_h.data_ptr(), xyz_h.data_ptr(), wl_h.data_ptr())
        for k in range(args.e2e_steps):
            if k + 1 < args.e2e_steps:
                pl.stage_host_ptr(T, S_h.data_ptr(), xyz_h.data_ptr(), wl_h.data_ptr())
            pl.reset()
            pl.process_staged()
            pl.images_ptr(img_h.data_ptr(), normalize=True, on_device=False)
        e1.record(stream)
        torch.cuda.synchronize()
        wall_e2e = time.perf_counter() - t0
        ems = torch.tensor([e0.elapsed_time(e1)], device=device, dtype=torch.float64)
        if world > 1:
            dist.all_reduce(ems, op=dist.ReduceOp.MAX)
        e2e = {"value": args.e2e_steps * T_steps * world / (float(ems.item()) / 1000.0), "unit": UNIT,
               "batches": args.e2e_steps, "host_wall_s": round(wall_e2e, 4),
               "copies": "staged (double-buffered): the first batch's copy is exposed, the later ones overlap",
               "h2d_bytes_per_step": int(lower_block_bytes(cfg.n_antenna, T) + xyz_h.numel() * 8 + wl_h.numel() * 8),
               "d2h_bytes_per_step": int(img_h.numel() * 4)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            Sc = S_h if not args.no_e2e else S  # noqa: F821
            v, cores, desc, extra = cpu_reference_sample(cfg, Sc, xyz, intervals, wl=float(wl[0].item()),
                                                         ref_eig_errors=True)
            cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "reference", "sample": desc,
                   "stages": "eigh_gram + virtual_vis", **extra}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": metric_of(args), "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded observation of the workload's shape, generated on the GPU)",
                "config": {"workload": workload_text(args),
                           "time_steps_per_batch": T_steps, "entries_per_batch": T, "mode": args.mode,
                           "vv_precision": args.vv_precision if args.mode == "batched" else "fp32",
                           "parallelism": f"dp{world} (steps)",
                           "l2": f"inputs ({S_bytes / 1e9:.1f} GB/batch) larger than L2; no flush"},
                "clocks": clk.summary(), "gpu_launches": gpu_launches, "stages_ms": stages, "e2e": e2e,
                "cpu_baseline": cpu, "roofline": roof, "plain_gpu": plain,
                "tuning": tuning,
                "image_rel_l2": parity and parity["image_rel_l2"],
                "eig_rel_err": parity and {
                    "per_eigenvalue_above_1e-2_of_max": parity["eig_rel_err_max_above_1e-2"],
                    "normwise": parity["eig_rel_err_normwise"],
                    "per_eigenvalue_all_in_level_range": parity["eig_rel_err_max"]},
                "parity": parity}
        print(json.dumps(line))
    pl.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
