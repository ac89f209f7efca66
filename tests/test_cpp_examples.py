"""The one-line switch on every example of the reference (no device): each examples/*.cpp with
SolverStatic<n_layer> -> SolverStaticGPU<n_layer> and SolverFatigue<n_layer> ->
SolverFatigueGPU<n_layer> (and the drop-in header included) compiles against the reference's own
headers and links against liblpmgpu.so.  The switched sources are written to a temporary
directory; nothing of the reference is copied into this repository.  Skipped where the reference
sources are not present (as on a GPU box)."""
import glob
import os
import re
import subprocess

import pytest

from _util import ROOT

# the LPM-CPP checkout: $LPM_REFERENCE, else a sibling directory "reference" of this repository
REF = os.environ.get("LPM_REFERENCE") or os.path.join(os.path.dirname(ROOT), "reference")
EXAMPLES = sorted(glob.glob(os.path.join(REF, "examples", "*.cpp")) +
                  glob.glob(os.path.join(REF, "examples", "plasticity", "*.cpp")))
LIBDIR = os.path.join(ROOT, "lpm-cpp_b200")


def _switch(src: str) -> str:
    out = re.sub(r"\bSolverStatic<n_layer>(\s)", r"SolverStaticGPU<n_layer>\1", src)
    out = re.sub(r"\bSolverFatigue<n_layer>(\s)", r"SolverFatigueGPU<n_layer>\1", out)
    header = "solver_fatigue_gpu.h" if "SolverFatigueGPU" in out else "solver_static_gpu.h"
    return re.sub(r"^void run\(\)", f'#include "{header}"\nvoid run()', out, count=1, flags=re.M)


@pytest.fixture(scope="module")
def shim_object(tmp_path_factory):
    """The MKL stand-in compiled once for all examples."""
    obj = str(tmp_path_factory.mktemp("shim") / "mkl_shim.o")
    subprocess.run(["g++", "-O0", "-fopenmp", "-std=c++17", "-DMKL_ILP64", "-w", "-c",
                    "-I", os.path.join(ROOT, "oracle", "shim"), os.path.join(ROOT, "oracle", "shim", "mkl_shim.cpp"),
                    "-o", obj], check=True)
    return obj


@pytest.mark.skipif(not EXAMPLES, reason="reference examples not present")
@pytest.mark.parametrize("path", EXAMPLES, ids=[os.path.basename(p)[:-4] for p in EXAMPLES])
def test_example_compiles_with_the_one_line_switch(path, tmp_path, shim_object):
    if not os.path.exists(os.path.join(LIBDIR, "liblpmgpu.so")):
        pytest.skip("liblpmgpu.so not built")
    src = open(path).read()
    switched = _switch(src)
    assert switched.count("GPU<n_layer>") >= 1, "the example constructs no solver"
    assert switched.replace("GPU<n_layer>", "<n_layer>").count("<n_layer>") == src.count("<n_layer>")
    name = os.path.basename(path)[:-4]
    (tmp_path / f"{name}.cpp").write_text(switched)
    (tmp_path / "main.cpp").write_text(f'#include "{name}.cpp"\nint main() {{ return 0; }}\n')
    cmd = ["g++", "-O0", "-fopenmp", "-std=c++17", "-DMKL_ILP64", "-w",
           "-I", os.path.join(ROOT, "oracle", "shim"), "-I", os.path.join(REF, "include"),
           "-I", os.path.join(LIBDIR, "cpp"), "-I", os.path.join(ROOT, "include"), "-I", str(tmp_path),
           "-o", str(tmp_path / "example"), str(tmp_path / "main.cpp"), shim_object, "-L", LIBDIR, "-llpmgpu"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
