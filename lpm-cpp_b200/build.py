"""Builds liblpmgpu.so (all CUDA sources in csrc/, sm_100a only) into this directory.

    python lpm-cpp_b200/build.py [--debug]

nvcc cross-compiles without a GPU.  -fmad=false keeps one rounding per operator so the bond,
force and exact stiffness kernels reproduce the reference's arithmetic exactly; the fast
assembly and the batched CG (CONTRACTED) are compiled with FMA.
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
# sources compiled with FMA contraction: the fast assembly, whose results are held to the
# reference within rounding instead of bit for bit, and the batched CG, whose members are held to
# their twins solved alone within tolerances (its partition already orders the sums differently)
CONTRACTED = {"assembly_fast.cu", "batch.cu"}


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


def _compile(args):
    cmd, src = args
    r = subprocess.run(cmd, capture_output=True, text=True)
    return src, r.returncode, r.stderr


def build(debug: bool = False, force: bool = False, verbose: bool = False) -> str:
    """Compiles every csrc/*.cu to an object in parallel (one nvcc per source, each its own
    translation unit as before) and links them into liblpmgpu.so."""
    if not force and not debug and up_to_date():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    objdir = os.path.join(HERE, "_build", "debug" if debug else "release")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-std=c++17", "-lineinfo", "-fmad=false", "-Xcompiler", "-fPIC", "-O0" if debug else "-O3"]
    if debug:
        flags.insert(0, "-DLPM_CHECK")
    if verbose:
        flags.insert(0, "-Xptxas=-v")
    jobs, objs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        f = flags
        if os.path.basename(src) in CONTRACTED:
            f = [x for x in flags if x != "-fmad=false"]
        jobs.append(([nvcc(), *f, "-c", "-o", obj, src], src))
    with ThreadPoolExecutor(max_workers=min(len(jobs), os.cpu_count() or 1)) as ex:
        results = list(ex.map(_compile, jobs))
    errs = [f"{os.path.basename(src)}:\n{err[-4000:]}" for src, rc, err in results if rc != 0]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    if verbose:
        for src, _, err in results:
            sys.stderr.write(f"== {os.path.basename(src)}\n{err}")
    r = subprocess.run([nvcc(), *ARCH, "-shared", "-o", OUT + ".tmp", *objs], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stderr[-6000:])
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(debug="--debug" in sys.argv, force=True, verbose="-v" in sys.argv))
