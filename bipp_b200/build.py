"""Build libbipp_b200.so in-tree with nvcc for sm_100a.

    python -m bipp_b200.build            # incremental
    python -m bipp_b200.build --force    # rebuild everything

Each .cu / .cpp under csrc/ is compiled to an object in _build/ and linked with
cuFFT into bipp_b200/libbipp_b200.so. No GPU is needed to build.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libbipp_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _flags():
    return ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
                   "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    inc = os.path.join(ROOT, "include")
    for dp, _, fs in os.walk(inc):
        hs += [os.path.join(dp, f) for f in fs]
    return hs


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = _sources()
    hmax = max((os.path.getmtime(h) for h in _headers()), default=0)
    objs, jobs = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hmax):
            jobs.append((s, o))

    def compile_one(job):
        s, o = job
        cmd = [nvcc()] + _flags() + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        return s, r

    failed = []
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for s, r in ex.map(compile_one, jobs):
            if r.returncode != 0:
                failed.append((s, r.stderr))
            elif verbose and r.stderr.strip():
                print(r.stderr)
    if failed:
        for s, err in failed:
            sys.stderr.write(f"--- {os.path.basename(s)}\n{err}\n")
        raise RuntimeError("nvcc failed for: " + ", ".join(os.path.basename(s) for s, _ in failed))
    if jobs or not os.path.exists(LIB):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcufft", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stderr)
            raise RuntimeError("link failed")
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose))


if __name__ == "__main__":
    main()
