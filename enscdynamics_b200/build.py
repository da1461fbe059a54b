"""Builds the sm_100a stepper library in-tree: enscdynamics_b200/_lib/libensc_b200.so.

Kernels that must reproduce the reference's FP64 arithmetic operation by
operation are compiled with ``-fmad=false`` (no multiply-add contraction);
the mixed-precision kernels allow contraction.  Usage::

    python -m enscdynamics_b200.build          # build if sources changed
    python -m enscdynamics_b200.build --force  # rebuild
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "_lib")
LIB = os.path.join(LIBDIR, "libensc_b200.so")
INCLUDE = os.path.join(ROOT, "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
          "--expt-relaxed-constexpr"]
# (source, extra flags)
UNITS = [
    ("ensc_fp64.cu", ["-fmad=false"]),
    ("ensc_control.cu", ["-fmad=false"]),
    ("ensc_mixed.cu", []),
    ("ensc_noalloc.cu", []),
    ("ensc_instance.cu", []),
    ("ensc_batch.cu", []),
    ("ensc_capi.cu", []),
]
HEADERS = ["ensc_device.cuh", "ensc_kernels.h", "ensc_instance.h"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _mtime(p: str) -> float:
    return os.path.getmtime(p) if os.path.exists(p) else -1.0


def _deps() -> List[str]:
    deps = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "ensc_gpu.h")]
    return [d for d in deps if os.path.exists(d)]


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    dep_time = max([_mtime(d) for d in _deps()] + [_mtime(__file__)])
    objs = []
    jobs = []
    for src, flags in UNITS:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or ptxas_info or _mtime(o) < max(_mtime(s), dep_time):
            cmd = [nvcc()] + ARCH + COMMON + flags + ["-c", s, "-o", o]
            if ptxas_info:
                cmd.insert(1, "-Xptxas=-v")
            jobs.append(cmd)
    procs = []
    for cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"nvcc failed: {' '.join(cmd)}\n{out}")
        if (verbose or ptxas_info) and out:
            print(out)
    if force or jobs or _mtime(LIB) < max(_mtime(o) for o in objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", tmp] + objs
        subprocess.run(cmd, check=True)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
