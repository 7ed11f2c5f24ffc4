"""Build libcansfz.so (sm_100a) in-tree with nvcc.

    python cans-fizzy_b200/build.py

The library lands next to the Python host package (cansfz/libcansfz.so) so
that the package loads it from the source tree.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SOURCES = ["csrc/k_stencil.cu", "csrc/k_tiles.cu", "csrc/k_momentum.cu", "csrc/k_init.cu", "csrc/k_bc.cu", "csrc/k_poisson.cu",
           "csrc/context.cu", "csrc/noalloc.cu", "csrc/k_xform_gemm.cu"]
OUT = os.path.join(HERE, "cansfz", "libcansfz.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
OBJDIR = os.path.join(HERE, "_build")


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build(force: bool = False, verbose: bool = False) -> str:
    srcs = [os.path.join(HERE, s) for s in SOURCES]
    deps = srcs + [os.path.join(HERE, "csrc", f) for f in os.listdir(os.path.join(HERE, "csrc"))]
    deps.append(os.path.join(os.path.dirname(HERE), "include", "cansfz.h"))
    if not force and os.path.exists(OUT):
        t = os.path.getmtime(OUT)
        if all(os.path.getmtime(d) <= t for d in deps if os.path.exists(d)):
            return OUT
    # one nvcc per source file, in parallel, then one link
    os.makedirs(OBJDIR, exist_ok=True)
    objs = [os.path.join(OBJDIR, os.path.basename(src)[:-3] + ".o") for src in srcs]
    procs = []
    for src, obj in zip(srcs, objs):
        cmd = [nvcc()] + ARCH + FLAGS + ["-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        procs.append((src, subprocess.Popen(cmd, cwd=HERE)))
    failed = [src for src, pr in procs if pr.wait() != 0]
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    cmd = [nvcc()] + ARCH + ["-shared", "-o", OUT] + objs
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=HERE)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
