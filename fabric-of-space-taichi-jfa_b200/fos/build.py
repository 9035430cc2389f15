"""Builds libfos.so in-tree for sm_100a with nvcc (no JIT, no fallback).

Flags: -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo -fmad=false.
-fmad=false keeps every FP32 expression in the reference's operator order
without FMA contraction (the parity-critical expressions also use explicit
__f*_rn intrinsics).  The static CUDA runtime is linked in.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT = os.path.join(HERE, "_lib", "libfos.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def sources() -> list[str]:
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def command(out: str = OUT, extra: list[str] | None = None) -> list[str]:
    return [nvcc(), *ARCH, "-O3", "-lineinfo", "-fmad=false", "-std=c++17", "-Xcompiler", "-fPIC",
            "-shared", f"-I{INCLUDE}", f"-I{CSRC}", *sources(), "-o", out, *(extra or [])]


def stale(out: str = OUT) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [os.path.join(INCLUDE, "fos.h")]
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    if force or stale():
        cmd = command()
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
