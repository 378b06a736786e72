"""Build libcuozblas_b200.so in-tree with nvcc for sm_100a.

    python ozblas_b200/build.py           (loads no package code, so it works
                                          before the library exists)

Every .cu/.cpp under ozblas_b200/csrc is compiled for
``-gencode arch=compute_100a,code=sm_100a`` and linked into one shared
library next to this file.  Object files go to ozblas_b200/_build/ and are
rebuilt only when a source or header is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libcuozblas_b200.so")
OBJDIR = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC,
         "--expt-relaxed-constexpr"]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))


def _headers():
    return glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(INCLUDE, "*.h"))


def build(verbose: bool = False, jobs: int = 8) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    hdr_mtime = max([os.path.getmtime(p) for p in _headers()] + [0])
    objs, cmds = [], []
    for src in _sources():
        obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_mtime):
            continue
        cmds.append([NVCC] + ARCH + FLAGS + ["-c", src, "-o", obj])
    procs = []
    for cmd in cmds:
        if verbose:
            print(" ".join(cmd))
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        if len(procs) >= jobs:
            _drain(procs)
    _drain(procs)
    need_link = not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs)
    if need_link:
        cmd = [NVCC] + ARCH + ["-shared", "-o", OUT] + objs + ["-lcudart"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stdout)
    return OUT


def _drain(procs):
    while procs:
        cmd, p = procs.pop(0)
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("nvcc failed: " + " ".join(cmd) + "\n" + out.decode(errors="replace"))
        elif out and os.environ.get("OZB_BUILD_VERBOSE"):
            sys.stdout.write(out.decode(errors="replace"))


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
