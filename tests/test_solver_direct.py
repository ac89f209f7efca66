"""The direct solver (lpmgpu_solve_direct, lpmgpu_desc.direct): the device's counterpart of the
reference's SolverMode::PARDISO (Solver::LPM_PARDISO, include/solver.h:191-274), a band Cholesky
after reverse Cuthill-McKee ordering.  Its arithmetic core is checked on the host against numpy
(tests/test_direct_host.py); here it runs on the device, through the C ABI.

Bars: one linear solve matches the tightly converged CG within 1e-9 relative; load paths solved
with it (K refactored whenever it is re-assembled, including the damage loop's re-assemblies)
match the tight-CG paths' Newton counts and displacements within 1e-9 relative, and the oracle's
within 1e-8; the Python SolverStatic with SolverMode.PARDISO takes it."""
import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, oracle_problem, oracle_step_args, rel

pytestmark = pytest.mark.gpu

TIGHT = dict(cg_rtol=1e-24, cg_atol=0.0)


def _cases():
    return {
        "hex": CFG.hex_plate(size=3.0, radius=0.1, steps=2, total_disp=0.002, tol_iter=1e-9),
        "sc": CFG.sc_cube(size=2.0, radius=0.2, steps=2, total_disp=0.002, tol_iter=1e-9),
        "hex_damage": CFG.hex_plate(size=2.0, radius=0.1, steps=3, total_disp=0.024, critical_bstrain=3e-3,
                                    tol_iter=1e-9),
    }


@pytest.mark.parametrize("name", ["hex", "sc"])
def test_direct_solve_matches_the_cg(name):
    case = _cases()[name]
    g = gpu_problem(case, **TIGHT)
    g.apply_load_step(case.load_step(0))
    g.update_force_state()  # the moved boundary particles' forces: a nonzero residual
    g.assemble(True)
    g.update_rr()
    xd, st = g.solve_direct()
    assert st["converged"] == 1 and st["cg_iters"] == 0
    xc, _ = g.solve_linear()
    assert np.linalg.norm(xc) > 0
    assert rel(xd, xc) <= 1e-9
    # a second solve reuses the factor and gives the same bits
    xd2, _ = g.solve_direct()
    assert np.array_equal(xd, xd2)
    g.close()


@pytest.mark.parametrize("name", ["hex", "sc", "hex_damage"])
def test_direct_newton_matches_the_cg_newton(name):
    case = _cases()[name]
    o = oracle_problem(case, **TIGHT)
    o.update_geometry()
    o.update_force_state()
    gd = LPM.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                        tol_iter=case.tol_iter, direct=1, **TIGHT)
    gc = gpu_problem(case, **TIGHT)
    for s in range(len(case.steps)):
        okd, sd = gd.solve_load_step(case.load_step(s))
        okc, sc = gc.solve_load_step(case.load_step(s))
        oko, so = o.solve_load_step(*oracle_step_args(case, s))
        assert okd and okc and oko
        assert sd["cg_iters"] == 0 and sd["newton_solves"] == sc["newton_solves"] == so["newton_solves"], s
        ud = gd.state(("xyz",))["xyz"] - case.xyz
        uc = gc.state(("xyz",))["xyz"] - case.xyz
        uo = o.state()["xyz"] - case.xyz
        assert rel(ud, uc) <= 1e-9, s
        assert rel(ud, uo) <= 1e-8, s
    if name == "hex_damage":
        assert (gd.state(("bdamage",))["bdamage"] == 1.0).any()
        assert np.array_equal(gd.state(("bdamage",))["bdamage"], gc.state(("bdamage",))["bdamage"])
    gd.close()
    gc.close()


def test_solver_static_pardiso_mode_solves_by_cg_first():
    """SolverMode.PARDISO runs the CG to a relative residual of 1e-12 (the band solve costs 20-58x
    the CG per load step on the benchmark plates) and keeps the band Cholesky for a system the CG
    cannot solve; the solution equals the tight CG's."""
    case = _cases()["hex"]
    solv = LPM.SolverStatic(case.undamaged_type, case.assembly(), LPM.StiffnessMode.Analytical,
                            LPM.SolverMode.PARDISO, "", case.max_iter, case.tol_iter)
    solv.solveProblem([case.load_step(s) for s in range(len(case.steps))], 0)
    assert all(h["cg_iters"] > 0 and h["newton_solves"] > 0 and h["direct_solves"] == 0 for h in solv.history)
    g = gpu_problem(case, **TIGHT)
    for s in range(len(case.steps)):
        g.solve_load_step(case.load_step(s))
    u = solv.problem.state(("xyz",))["xyz"] - case.xyz
    assert rel(u, g.state(("xyz",))["xyz"] - case.xyz) <= 1e-9
    g.close()


@pytest.mark.parametrize("name", ["hex", "hex_damage"])
def test_solver_static_gpu_pardiso_matches_the_reference(name, tmp_path):
    """SolverStaticGPU with SolverMode::PARDISO (the device CG at 1e-12, the band Cholesky behind it) against the
    reference's SolverStatic with SolverMode::PARDISO (Solver::LPM_PARDISO; the MKL stand-in's
    PARDISO solves to 1e-14): the same driver built both ways.  Per step: displacements within
    1e-8 relative and the same broken bonds."""
    import os
    from _util import O
    for b in (O.REF_BIN, O.REF_GPU_BIN):
        if not os.path.exists(b):
            pytest.skip(f"{os.path.basename(b)} not built (make -C oracle ref ref-gpu)")
    case = _cases()[name]
    out = {}
    for tag, binary in (("cpu", O.REF_BIN), ("gpu", O.REF_GPU_BIN)):
        d = str(tmp_path / tag)
        O.run_ref(O.write_ref_spec(case, d, loop="ref", solver="pardiso"), d, threads=1, timeout=900, binary=binary)
        out[tag] = d
    x0 = O.read_bin(out["cpu"], "xyz0.f64", np.float64)
    rc, rg = O.read_ref_steps(out["cpu"]), O.read_ref_steps(out["gpu"])
    assert len(rc) == len(rg) == len(case.steps)
    for s in range(len(case.steps)):
        t = f"{s:03d}"
        uc = O.read_bin(out["cpu"], f"xyz_{t}.f64", np.float64) - x0
        ug = O.read_bin(out["gpu"], f"xyz_{t}.f64", np.float64) - x0
        assert rel(ug, uc) <= 1e-8, s
        bc = O.read_bin(out["cpu"], f"bdamage_{t}.f64", np.float64)
        bg = O.read_bin(out["gpu"], f"bdamage_{t}.f64", np.float64)
        assert np.array_equal(bc == 1.0, bg == 1.0), s
        assert rc[s]["cuts"] == rg[s]["cuts"] == 0


def test_pardiso_mode_falls_back_to_the_band_solve_when_the_cg_fails():
    """desc.direct = 2 with a CG cap too small to converge: every Newton solve's CG stops at its
    cap and the band Cholesky solves the system instead; the load path equals the direct path's."""
    case = _cases()["hex"]
    gf = LPM.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                        tol_iter=case.tol_iter, direct=2, cg_maxit=3, **TIGHT)
    gd = LPM.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter,
                        tol_iter=case.tol_iter, direct=1, **TIGHT)
    for s in range(len(case.steps)):
        okf, sf = gf.solve_load_step(case.load_step(s))
        okd, sd = gd.solve_load_step(case.load_step(s))
        assert okf and okd
        assert sf["direct_solves"] == sf["newton_solves"] == sd["newton_solves"] == sd["direct_solves"], (s, sf, sd)
        assert sf["cg_maxit_hits"] == sf["newton_solves"]
        uf = gf.state(("xyz",))["xyz"] - case.xyz
        ud = gd.state(("xyz",))["xyz"] - case.xyz
        assert rel(uf, ud) <= 1e-12, s
    gf.close()
    gd.close()
