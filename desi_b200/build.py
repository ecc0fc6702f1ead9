"""Compile libpcf.so (and the PCF.out drop-in CLI) for sm_100a, in tree.

Run as ``python -m desi_b200.build`` or through ``__graft_entry__.build()``.
nvcc cross-compiles for sm_100a without a GPU.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libpcf.so")
CLI = os.path.join(PKG, "PCF.out")
OBJ = os.path.join(PKG, "_build")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--fmad=true",
         "-I", os.path.join(ROOT, "include")]


def _run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    cu = sorted(glob.glob(os.path.join(CSRC, "*.cu"))) + [
        s for s in sorted(glob.glob(os.path.join(CSRC, "*.cpp"))) if not s.endswith("pcf_main.cpp")]
    hdr = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(ROOT, "include", "*.h"))
    lib_src = [s for s in cu if not s.endswith("pcf_main.cu")]
    if force or _stale(LIB, lib_src + hdr):
        # one object per source, compiled in parallel, then one link
        extra = ["-Xptxas", "-v"] if verbose_ptxas else []
        os.makedirs(OBJ, exist_ok=True)
        objs = [os.path.join(OBJ, os.path.basename(s) + ".o") for s in lib_src]
        todo = [(s, o) for s, o in zip(lib_src, objs) if force or _stale(o, [s] + hdr)]
        with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 4))) as ex:
            list(ex.map(lambda so: _run([NVCC, *ARCH, *FLAGS, *extra, "-c", "-o", so[1], so[0]]),
                        todo))
        _run([NVCC, *ARCH, "-shared", "-o", LIB, *objs])
    cli_src = os.path.join(CSRC, "pcf_main.cpp")
    if os.path.exists(cli_src) and (force or _stale(CLI, [cli_src, LIB] + hdr)):
        _run([NVCC, *ARCH, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
              "-o", CLI, cli_src, "-L", PKG, "-lpcf", "-Xlinker", "-rpath,$ORIGIN"])
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose_ptxas="-v" in sys.argv)
