"""Build recipe for libdftcuda.so (sm_100a) from csrc/, in place next to this file.

Run as ``python dft-zig_b200/build.py`` or through ``__graft_entry__.build()``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I" + os.path.join(ROOT, "include")]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def build(verbose: bool = False, force: bool = False) -> str:
    out = os.path.join(HERE, "libdftcuda.so")
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "dftcuda.h")]
    if not force and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(p) for p in deps):
        return out
    cmd = [NVCC, *ARCH, *FLAGS, "-o", out, *srcs]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libdftcuda.so")
    return out


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
