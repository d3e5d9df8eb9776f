"""Builds libllalbm_cuda.so in-tree with nvcc for sm_100a.

    python build.py            # incremental
    python build.py --force    # rebuild everything

The FP64 kernels (csrc/llb_f64.cu) are compiled with --fmad=false so their
arithmetic rounds exactly like the reference's x86-64 build.  The shifted
low-precision kernels (csrc/llb_lowp.cu) are compiled the same way and write
their multiply-adds out (__fmaf_rn), so every kernel of a form rounds alike.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libllalbm_cuda.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-I", CSRC, "-I", INCLUDE]

SOURCES = {
    "llb_f64.cu": ["--fmad=false"],
    "llb_lowp.cu": ["--fmad=false"],
    "llb_capi.cu": [],
    "llb_noalloc.cu": [],
    "llb_batch.cu": [],
    "llb_server.cpp": [],
    "llb_classify.cpp": [],
    "llb_writer.cpp": [],
}
HEADERS = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))] + [
    os.path.join(INCLUDE, "llalbm_cuda.h")
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    objs = []
    relinked = force
    for src, extra in SOURCES.items():
        path = os.path.join(CSRC, src)
        obj = os.path.join(OBJ, src + ".o")
        objs.append(obj)
        if force or _stale(obj, [path, *HEADERS, __file__]):
            lang = ["-x", "cu"] if src.endswith(".cu") else []
            cmd = [nvcc(), *ARCH, *COMMON, *extra, *lang, "-c", path, "-o", obj]
            if verbose:
                print(" ".join(cmd))
            subprocess.check_call(cmd)
            relinked = True
    if relinked or _stale(LIB, objs):
        tmp = LIB + ".tmp"
        cmd = [nvcc(), *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
        if verbose:
            print(" ".join(cmd))
        subprocess.check_call(cmd)
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.v))
    sys.exit(0)
