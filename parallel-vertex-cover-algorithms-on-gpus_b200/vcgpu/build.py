"""Build recipe for the native parts, in-tree.

  libvcgpu.so  -- the solver library (C ABI in include/vcgpu.h), sm_100a only
  output       -- the reference-compatible command line (`./output <args>`)

Both land in the package directory so they travel with the source tree.
Each product is rebuilt unless the SHA-256 of its compile command and of every
source and header it depends on equals the one recorded beside it when it was
built (`<product>.srchash`): a prebuilt file is reused only for exactly these
sources, whatever the file times say.
"""
from __future__ import annotations

import glob
import hashlib
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


def _digest(cmd, sources) -> str:
    """Independent of where the tree lives (paths are taken relative to it)."""
    h = hashlib.sha256(" ".join(c.replace(REPO, ".") for c in cmd).encode())
    for path in sorted(sources):
        h.update(os.path.relpath(path, REPO).encode())
        with open(path, "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def _stale(product: str, digest: str) -> bool:
    if not os.path.exists(product) or not os.path.exists(product + ".srchash"):
        return True
    with open(product + ".srchash") as f:
        return f.read().strip() != digest


def _record(product: str, digest: str) -> None:
    with open(product + ".srchash", "w") as f:
        f.write(digest + "\n")


def lib_sources():
    return sorted(glob.glob(os.path.join(CSRC, "vc_*.cu")) + glob.glob(os.path.join(CSRC, "vc_*.cpp")))


def build(force: bool = False, verbose: bool = False) -> None:
    srcs = lib_sources()
    deps = srcs + glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(REPO, "include", "vcgpu.h")]
    nvcc = _nvcc()
    cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-shared", "-o", LIB] + srcs
    dig = _digest([os.path.basename(c) if c == nvcc else c for c in cmd], deps)
    if force or _stale(LIB, dig):
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        _record(LIB, dig)
    main_src = os.path.join(CSRC, "main.cpp")
    if os.path.exists(main_src):
        cmd = [nvcc] + ARCH + NVCC_FLAGS + ["-o", CLI, main_src, "-L" + PKG, "-lvcgpu",
                                            "-Xlinker", "-rpath,$ORIGIN"]
        dig_cli = _digest([os.path.basename(c) if c == nvcc else c for c in cmd] + [dig], deps + [main_src])
        if force or _stale(CLI, dig_cli):
            if verbose:
                print(" ".join(cmd), file=sys.stderr)
            subprocess.run(cmd, check=True)
            _record(CLI, dig_cli)


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
