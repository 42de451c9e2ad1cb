"""Builds libipg.so (the C-ABI library) for sm_100a, in-tree.

    python interatomicpotentials.jl_b200/build.py [--verbose] [--ptxas]

Every .cu file directly under csrc/ is compiled with nvcc
(-gencode arch=compute_100a,code=sm_100a) in parallel and linked into
interatomicpotentials.jl_b200/ipg/libipg.so with a static CUDA runtime; the FP64 peak
probe (csrc/probe/fp64_peak.cu, a measurement tool for bench.py) is built into
ipg/libipg_probe.so.  Object files go
to interatomicpotentials.jl_b200/_build/.  A file is recompiled only when it, or a header
it includes, is newer than its object.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
OUT = os.path.join(HERE, "ipg", "libipg.so")
PROBE_SRC = os.path.join(CSRC, "probe", "fp64_peak.cu")
PROBE_OUT = os.path.join(HERE, "ipg", "libipg_probe.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-DIPG_BUILD"]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(ROOT, "include", "ipg.h")]


def _stale(src, obj, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return os.path.getmtime(src) > m or hdr_mtime > m


def build(verbose=False, ptxas=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(BUILD, os.path.basename(s) + ".o")
        objs.append(o)
        if force or _stale(s, o, hdr_mtime):
            cmd = [NVCC, *ARCH, *FLAGS, "-c", s, "-o", o]
            if ptxas and s.endswith(".cu"):
                cmd += ["-Xptxas", "-v"]
            if s.endswith(".cpp"):
                cmd = [NVCC, *FLAGS, "-c", s, "-o", o]
            jobs.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    ok = True
    with cf.ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, r in ex.map(run, jobs):
            if verbose or r.returncode or ptxas:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            ok &= r.returncode == 0
    if not ok:
        raise RuntimeError("nvcc compilation failed")
    if jobs or not os.path.exists(OUT):
        cmd = [NVCC, *ARCH, "-shared", "-cudart", "static", "-o", OUT, *objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError("link failed")
    if force or not os.path.exists(PROBE_OUT) or os.path.getmtime(PROBE_SRC) > os.path.getmtime(PROBE_OUT):
        cmd = [NVCC, *ARCH, "-O3", "-shared", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
               "-cudart", "static", "-o", PROBE_OUT, PROBE_SRC]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if verbose or r.returncode:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        if r.returncode:
            raise RuntimeError("probe build failed")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print -Xptxas -v resource usage")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.ptxas, a.force))
