"""Builds the CUDA library libqbx.so in-tree (qbox-public_b200/qbx/) for sm_100a.

    python qbox-public_b200/qbx/build.py

nvcc compiles every source under qbox-public_b200/csrc with
-gencode arch=compute_100a,code=sm_100a and links cuBLAS and cuSOLVER.
Objects are rebuilt only when a source or header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OBJDIR = os.path.join(PKG, "_build")
LIB = os.path.join(HERE, "libqbx.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3",
         "-I" + CSRC, "-I" + os.path.join(ROOT, "include"),
         "--expt-relaxed-constexpr"]


def _newer(src, dst):
    return not os.path.exists(dst) or os.path.getmtime(src) > os.path.getmtime(dst)


def build(verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    headers = (glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh"))
               + [os.path.join(ROOT, "include", "qbx.h")])
    hdr_time = max(os.path.getmtime(h) for h in headers)
    objs = []
    procs = []
    for src in sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp"))):
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if _newer(src, obj) or hdr_time > os.path.getmtime(obj):
            cmd = [NVCC] + ARCH + FLAGS + ["-x", "cu" if src.endswith(".cu") else "c++",
                                          "-c", src, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out))
        elif verbose and out.strip():
            print(out)
    if failed:
        for src, out in failed:
            sys.stderr.write(f"--- {src}\n{out}\n")
        raise RuntimeError("nvcc failed")
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L/usr/local/cuda/lib64", "-lcublas", "-lcusolver", "-lcudart",
            "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
