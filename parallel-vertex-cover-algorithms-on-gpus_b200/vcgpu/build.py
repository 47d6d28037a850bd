"""Build recipe for the native parts, in-tree.

  libvcgpu.so  -- the solver library (C ABI in include/vcgpu.h), sm_100a only
  output       -- the reference-compatible command line (`./output <args>`)

Both land in the package directory so they travel with the source tree.
Rebuilds only when a source is newer than its product.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libvcgpu.so")
CLI = os.path.join(PKG, "output")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + os.path.join(REPO, "include")]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(product: str, sources) -> bool:
    if not os.path.exists(product):
        return True
    t = os.path.getmtime(product)
    return any(os.path.getmtime(s) > t for s in sources)


def lib_sources():
    return sorted(glob.glob(os.path.join(CSRC, "vc_*.cu")) + glob.glob(os.path.join(CSRC, "vc_*.cpp")))


def build(force: bool = False, verbose: bool = False) -> None:
    srcs = lib_sources()
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(REPO, "include", "vcgpu.h")]
    nvcc = _nvcc()
    if force or _stale(LIB, deps):
        cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-shared", "-o", LIB] + srcs
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
    main_src = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main_src) and (force or _stale(CLI, [main_src, LIB] + deps)):
        cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-o", CLI, main_src, "-L" + PKG, "-lvcgpu",
                                            "-Xlinker", "-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
