"""Builds core_b200/libunwrap_b200.so from core_b200/csrc with nvcc for sm_100a.

    python -m core_b200._build [--debug] [--jobs N]

Each .cu file is compiled separately (in parallel) and linked into one shared
library with the CUDA runtime linked statically, so the library does not depend
on which libcudart the host process has loaded.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
OUT = os.path.join(PKG, "libunwrap_b200.so")
BUILD = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _flags(debug):
    f = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fvisibility=hidden", "--expt-relaxed-constexpr",
         "-I" + os.path.join(os.path.dirname(PKG), "include")]
    if debug:
        f += ["-DUNW_CHECKS=1"]
    return ARCH + f


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def build(debug=False, jobs=None, verbose=False, ptxas_v=False):
    os.makedirs(BUILD, exist_ok=True)
    objs = []
    cmds = []
    for src in sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        cmd = [NVCC] + _flags(debug) + (["-Xptxas", "-v"] if ptxas_v else []) + ["-c", src, "-o", obj]
        cmds.append(cmd)

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        for cmd, r in ex.map(run, cmds):
            if verbose or r.returncode != 0 or ptxas_v:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode != 0:
                raise RuntimeError("nvcc failed: " + " ".join(cmd))
    link = [NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", OUT] + objs
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout + r.stderr)
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--debug", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--ptxas-v", action="store_true")
    a = ap.parse_args()
    print(build(debug=a.debug, jobs=a.jobs, verbose=True, ptxas_v=a.ptxas_v))
