"""The C++ drop-in SolverStaticGPU (lpm-cpp_b200/cpp/solver_static_gpu.h) against SolverStatic.

Both binaries are the same driver (oracle/ref_driver.cpp) compiled from the reference's own
headers; lpm_ref_gpu differs only by the one-line switch SolverStatic -> SolverStaticGPU.
The reference's Assembly, Particle, LoadStep and DispBC/ForceBC objects therefore feed the device
library exactly as an LPM-CPP example would, and the loop is SolverStatic::solveProblem's
(halve-and-retry included, solver_static.h:65-96).  Both sides solve tightly (CG squared-norm
test 1e-24 relative, Newton 1e-9), so per step: Newton solves and load cuts equal, displacements
within 1e-8 relative, broken-bond sets equal, the exported stiffness pattern bit-exact and its
values within 1e-9 of max|K|.
"""
import os

import numpy as np
import pytest

from _util import CFG, LPM, O, hetero_plate, rel

pytestmark = pytest.mark.gpu

DISP_TOL = 1e-8
K_TOL = 1e-9
TIGHT = dict(cg_tol=(1e-24, 0.0), tol_iter=1e-9, loop="ref")


def _need_binaries():
    for b in (O.REF_BIN, O.REF_GPU_BIN):
        if not os.path.exists(b):
            pytest.skip(f"{os.path.basename(b)} not built (make -C oracle ref ref-gpu)")


def _cases():
    return {
        "hex": (CFG.hex_plate(size=3.0, radius=0.1, steps=3, total_disp=0.003), {}),
        "sc_j2": (CFG.sc_cube(size=2.0, radius=0.25, steps=3, total_disp=0.06,
                              ptype=LPM.ParticleType.J2Plasticity, j2=(200.0, 0.0, 38714.0, 10.0)), {}),
        "hex_damage": (CFG.hex_plate(size=2.0, radius=0.1, steps=3, total_disp=0.024, critical_bstrain=3e-3), {}),
        # pre-crack: both binaries build the Assembly through readDump + readBond
        "hex_crack": (CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=6, total_disp=0.006), {}),
        # per-bond Kn/Tv and initial bond damage set in the reference's Bond objects
        "hex_hetero": (hetero_plate(), {}),
        # a Newton cap of 5 makes the full step fail, so solveProblem halves it
        "hex_cut": (CFG.hex_plate(size=2.0, radius=0.1, steps=1, total_disp=0.01), {"max_iter": 5}),
    }


CASES = _cases()


@pytest.mark.parametrize("name", sorted(CASES))
def test_solver_static_gpu_matches_solver_static(name, tmp_path):
    _need_binaries()
    case, extra = CASES[name]
    nsteps = len(case.steps)
    out = {}
    for tag, binary in (("cpu", O.REF_BIN), ("gpu", O.REF_GPU_BIN)):
        d = str(tmp_path / tag)
        spec = O.write_ref_spec(case, d, dump_k=(nsteps - 1,), **TIGHT, **extra)
        # one thread: the MKL stand-in's SpMV then sums in one fixed order, as in the golden runs
        O.run_ref(spec, d, threads=1, timeout=900, binary=binary)
        out[tag] = d
    rc, rg = O.read_ref_steps(out["cpu"]), O.read_ref_steps(out["gpu"])
    assert len(rc) == len(rg) == nsteps
    x0 = O.read_bin(out["cpu"], "xyz0.f64", np.float64)
    assert np.array_equal(x0, O.read_bin(out["gpu"], "xyz0.f64", np.float64))
    for s in range(nsteps):
        assert rc[s]["cuts"] == rg[s]["cuts"], f"step {s}: load cuts {rc[s]['cuts']} vs {rg[s]['cuts']}"
        assert rc[s]["newton_solves"] == rg[s]["newton_solves"], f"step {s}: Newton solves differ"
        t = f"{s:03d}"
        uc = O.read_bin(out["cpu"], f"xyz_{t}.f64", np.float64) - x0
        ug = O.read_bin(out["gpu"], f"xyz_{t}.f64", np.float64) - x0
        assert rel(ug, uc) <= DISP_TOL, f"step {s}: displacement rel err {rel(ug, uc)}"
        bc = O.read_bin(out["cpu"], f"bdamage_{t}.f64", np.float64)
        bg = O.read_bin(out["gpu"], f"bdamage_{t}.f64", np.float64)
        assert np.array_equal(bc == 1.0, bg == 1.0), f"step {s}: broken bond sets differ"
        svc = O.read_bin(out["cpu"], f"state_var_{t}.f64", np.float64)
        svg = O.read_bin(out["gpu"], f"state_var_{t}.f64", np.float64)
        assert svc.shape == svg.shape
        if svc.size and np.linalg.norm(svc) > 0:
            assert rel(svg, svc) <= 100 * DISP_TOL, f"step {s}: state_var rel err {rel(svg, svc)}"
    if name in ("hex_damage", "hex_crack"):
        assert (O.read_bin(out["cpu"], f"bdamage_{nsteps - 1:03d}.f64", np.float64) == 1.0).any()
    if name == "hex_cut":
        assert rc[0]["cuts"] > 0
    t = f"{nsteps - 1:03d}"
    for f in ("K_pointer", "IK", "JK"):
        a = O.read_bin(out["cpu"], f"{f}_{t}.i64", np.int64)
        b = O.read_bin(out["gpu"], f"{f}_{t}.i64", np.int64)
        assert np.array_equal(a, b), f"{f} differs"
    kc = O.read_bin(out["cpu"], f"K_{t}.f64", np.float64)
    kg = O.read_bin(out["gpu"], f"K_{t}.f64", np.float64)
    err = np.abs(kg - kc).max() / np.abs(kc).max()
    assert err <= K_TOL, f"stiffness max err {err} of max|K|"
