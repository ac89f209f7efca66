"""Reference examples run end to end through the one-line switch.  oracle/Makefile (target
examples) builds examples/ex7_convergence_beam.cpp and examples/ex1_isoelasticity_2d_hex.cpp twice
from the reference's sources: as they are (the reference's SolverStatic, MKL replaced by the
oracle/shim stand-in) and with SolverStatic<n_layer> -> SolverStaticGPU<n_layer>.  Both run in
their own directories and write the files the examples write; the device build's must match.

Bars: the printed L2 error of the beam (the reference's known answer, solution.h:27-63) equal to
its printed digits; the beam's approximate solution within 1e-6 of its largest entry; ex1's
exported matrix pattern (K_pointer, IK, JK) identical as text and its values within 2e-5 of
max|K| (printed with 6 digits); the dumps' displacements within 1e-3 of their largest (printed
with 5 digits)."""
import os
import subprocess

import numpy as np
import pytest

from _util import ROOT

pytestmark = pytest.mark.gpu

REF_DIR = os.path.join(ROOT, "oracle", "_ref")


def _run(name, tag, cwd):
    exe = os.path.join(REF_DIR, f"{name}_{tag}")
    if not os.path.exists(exe):
        pytest.skip(f"{os.path.basename(exe)} not built (make -C oracle examples)")
    os.makedirs(cwd, exist_ok=True)
    env = dict(os.environ, OMP_NUM_THREADS="1")
    r = subprocess.run([exe], cwd=cwd, env=env, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stdout


def _dump_disp(path):
    lines = open(path).read().splitlines()
    n = int(lines[3])
    rows = np.array([ln.split()[5:8] for ln in lines[9:9 + n]], dtype=float)
    return rows


def test_beam_example_through_the_switch(tmp_path):
    out = {}
    for tag in ("cpu", "gpu"):
        d = str(tmp_path / tag)
        stdout = _run("ex7_convergence_beam", tag, d)
        out[tag] = ([ln for ln in stdout.splitlines() if ln.startswith("L2 error is:")],
                    np.loadtxt(os.path.join(d, "approx_sol.txt")), _dump_disp(os.path.join(d, "beam_convergence.dump")))
    assert out["cpu"][0] == out["gpu"][0] and out["cpu"][0], (out["cpu"][0], out["gpu"][0])
    a, b = out["cpu"][1], out["gpu"][1]
    assert np.abs(a - b).max() <= 1e-6 * np.abs(a).max()
    assert np.abs(out["cpu"][2] - out["gpu"][2]).max() <= 1e-3 * np.abs(out["cpu"][2]).max()


def test_hex_example_through_the_switch(tmp_path):
    dirs = {}
    for tag in ("cpu", "gpu"):
        dirs[tag] = str(tmp_path / tag)
        _run("ex1_isoelasticity_2d_hex", tag, dirs[tag])
    for f in ("matrix_K_pointer.txt", "matrix_IK.txt", "matrix_JK.txt"):
        assert open(os.path.join(dirs["cpu"], f)).read() == open(os.path.join(dirs["gpu"], f)).read(), f
    kc = np.loadtxt(os.path.join(dirs["cpu"], "matrix_K_global.txt"))
    kg = np.loadtxt(os.path.join(dirs["gpu"], "matrix_K_global.txt"))
    assert kc.shape == kg.shape and np.abs(kc - kg).max() <= 2e-5 * np.abs(kc).max()
    uc = _dump_disp(os.path.join(dirs["cpu"], "hex_position.dump"))
    ug = _dump_disp(os.path.join(dirs["gpu"], "hex_position.dump"))
    assert np.abs(uc - ug).max() <= 1e-3 * np.abs(uc).max()


def test_fcc_pardiso_example_through_the_switch(tmp_path):
    """examples/ex3_singlecrystal_3d_fcc.cpp: 10,976 FCC particles, elastic with cubic constants
    (C11, C12, C44) and a brittle bond law, solved in SolverMode::PARDISO, which the drop-in runs as
    the device's direct solve where its band fits (else the CG to 1e-12); the reference's PARDISO
    stand-in solves to 1e-14."""
    dirs = {}
    for tag in ("cpu", "gpu"):
        dirs[tag] = str(tmp_path / tag)
        _run("ex3_singlecrystal_3d_fcc", tag, dirs[tag])
    uc = _dump_disp(os.path.join(dirs["cpu"], "Crystal_position.dump"))
    ug = _dump_disp(os.path.join(dirs["gpu"], "Crystal_position.dump"))
    assert uc.shape == ug.shape and np.abs(uc).max() > 0
    assert np.abs(uc - ug).max() <= 1e-3 * np.abs(uc).max()
