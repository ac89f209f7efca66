"""Builds liblpmgpu.so (all CUDA sources in csrc/, sm_100a only) into this directory.

    python lpm-cpp_b200/build.py [--debug]

nvcc cross-compiles without a GPU.  -fmad=false keeps one rounding per operator so the bond,
force and stiffness kernels reproduce the reference's arithmetic exactly.
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "liblpmgpu.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def up_to_date() -> bool:
    if not os.path.exists(OUT):
        return False
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(HERE, "csrc", "*.cuh")) + [
        os.path.join(HERE, "..", "include", "lpmgpu.h")]
    return all(os.path.getmtime(d) <= t for d in deps)


def build(debug: bool = False, force: bool = False, verbose: bool = False) -> str:
    if not force and not debug and up_to_date():
        return OUT
    cmd = [nvcc(), *ARCH, "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-shared",
           "-O0" if debug else "-O3", "-o", OUT + ".tmp", *sources()]
    if debug:
        cmd.insert(1, "-DLPM_CHECK")
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-6000:])
    os.replace(OUT + ".tmp", OUT)
    if verbose:
        sys.stderr.write(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, force=True, verbose="-v" in sys.argv))
