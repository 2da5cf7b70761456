"""Build the in-tree CUDA library ``lzx_b200/_build/liblattice_cuda.so`` for sm_100a.

``python -m lzx_b200.build`` or :func:`build`.  nvcc cross-compiles without a
GPU; the resulting .so travels with the source tree.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT = os.path.join(HERE, "_build", "liblattice_cuda.so")
SOURCES = sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))
DEPS = SOURCES + sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + \
    sorted(glob.glob(os.path.join(HERE, "csrc", "*.h"))) + \
    sorted(glob.glob(os.path.join(ROOT, "include", "*.h")))

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-shared",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    return all(os.path.getmtime(d) <= t for d in DEPS)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    tmp = OUT + ".tmp"
    # separate objects compiled in parallel, then linked into one shared library
    objs = []
    procs = []
    for src in SOURCES:
        obj = os.path.join(os.path.dirname(OUT), os.path.basename(src) + ".o")
        objs.append(obj)
        cmd = [_nvcc()] + [f for f in NVCC_FLAGS if f != "-shared"] + ["-c", src, "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + out.decode(errors="replace"))
        if verbose and out:
            print(out.decode(errors="replace"))
    link = [_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", tmp] + objs
    subprocess.run(link, check=True)
    os.replace(tmp, OUT)
    for o in objs:
        os.remove(o)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
