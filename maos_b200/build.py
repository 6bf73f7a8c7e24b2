"""Build recipe for the native library of the B200 Shack-Hartmann frame.

Compiles maos_b200/csrc/*.cu with nvcc for sm_100a and the host setup code
(maos_b200/csrc/host/*.c) with gcc, linked into
maos_b200/libshwfs_b200.so (in-tree, so the built library travels with the
source tree).  Run as ``python -m maos_b200.build``.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libshwfs_b200.so")
SOURCES = [os.path.join(HERE, "csrc", "shwfs_api.cu")]
HOST_SOURCES = [os.path.join(HERE, "csrc", "host", f) for f in ("hmath.c", "setup.c", "binio.c")]
OBJDIR = os.path.join(HERE, "_build")


def _deps():
    out = []
    for d in (os.path.join(HERE, "csrc"), os.path.join(HERE, "csrc", "host"), os.path.join(ROOT, "include")):
        out += [os.path.join(d, f) for f in os.listdir(d) if not os.path.isdir(os.path.join(d, f))]
    return out

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return LIB
    os.makedirs(OBJDIR, exist_ok=True)
    objs = []
    for src in HOST_SOURCES:
        obj = os.path.join(OBJDIR, os.path.basename(src)[:-2] + ".o")
        subprocess.run([os.environ.get("CC", "gcc"), "-std=gnu11", "-O2", "-fPIC", "-Wall", "-Wno-unused-function",
                        "-c", src, "-o", obj], check=True)
        objs.append(obj)
    cmd = [nvcc(), *NVCC_FLAGS, *SOURCES, *objs, "-lz", "-o", LIB]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
