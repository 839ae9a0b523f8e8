"""Builds the native library in-tree: open_source_einstar_b200/lib/libdepth_cuda.so (sm_100a).

nvcc cross-compiles without a GPU. The library links the CUDA runtime statically, so the .so loads on
any machine with a CUDA driver and nothing else from this image.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB_DIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIB_DIR, "libdepth_cuda.so")

# -fmad=false: every float operation of this library is meant to round separately, as the reference's x86-64
# build evaluates it; no plain multiply and add may be contracted into a fused multiply-add.
NVCC_FLAGS = [
    "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
    "-Xcompiler", "-fPIC,-fvisibility=hidden", "-shared", "-cudart", "static",
]

SOURCES = ["depth_cuda.cu", "noalloc.cu", "server.cu", "points.cu", "recording.cu", "sweep_cols.cu", "sweep_rows.cu", "wta.cu", "inst_r1.cu", "inst_r2.cu", "inst_r3.cu", "inst_r4.cu", "inst_r6.cu", "inst_r8.cu"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return "nvcc"


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_native(force: bool = False, verbose: bool = False) -> str:
    """Compiles libdepth_cuda.so when any source or header is newer than it."""
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "depth_cuda.h")]
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    obj_dir = os.path.join(PKG, "_build")
    os.makedirs(obj_dir, exist_ok=True)
    compile_flags = [f for f in NVCC_FLAGS if f not in ("-shared",)]
    procs, objs = [], []
    for src in SOURCES:
        obj = os.path.join(obj_dir, src.replace(".cu", ".o"))
        objs.append(obj)
        cmd = [_nvcc(), *compile_flags, "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        procs.append((src, subprocess.Popen(cmd)))
    failed = [src for src, p in procs if p.wait() != 0]
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", LIB, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build_native(force="--force" in sys.argv, verbose=True))
