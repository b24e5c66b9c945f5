"""Build recipe for libdftcuda.so (sm_100a) from csrc/, in place next to this file.

Each translation unit compiles to its own object under _build/ (in parallel, one nvcc per source;
a source is recompiled when it, or any shared header, is newer than its object), then the objects
are linked into the shared library.  Run as ``python dft-zig_b200/build.py`` or through
``__graft_entry__.build()``.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(ROOT, "include")]
OBJDIR = os.path.join(HERE, "_build")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def _headers():
    return glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [os.path.join(ROOT, "include", "dftcuda.h")]


def _compile(src: str, obj: str, verbose: bool):
    cmd = [NVCC, *ARCH, *FLAGS, "-c", "-o", obj, src]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stdout + r.stderr


def build(verbose: bool = False, force: bool = False) -> str:
    out = os.path.join(HERE, "libdftcuda.so")
    srcs = sources()
    hdr_time = max(os.path.getmtime(p) for p in _headers())
    os.makedirs(OBJDIR, exist_ok=True)
    objs, todo = [], []
    for s in srcs:
        o = os.path.join(OBJDIR, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), hdr_time):
            todo.append((s, o))
    if todo:
        with ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            results = list(ex.map(lambda so: _compile(so[0], so[1], verbose), todo))
        bad = [(s, log) for s, rc, log in results if rc != 0]
        for s, rc, log in results:
            if log.strip() and (verbose or rc != 0):
                sys.stderr.write(log)
        if bad:
            for _, o in todo:
                if os.path.exists(o) and any(o.endswith(os.path.basename(s)[:-3] + ".o") for s, _ in bad):
                    os.remove(o)
            raise RuntimeError("nvcc failed building libdftcuda.so: " + ", ".join(os.path.basename(s) for s, _ in bad))
    if todo or not os.path.exists(out) or os.path.getmtime(out) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", out, *objs]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(r.stdout + r.stderr)
            raise RuntimeError("nvcc failed linking libdftcuda.so")
    return out


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="--force" in sys.argv))
