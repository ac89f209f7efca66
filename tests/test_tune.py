"""The CG launch-shape autotuner (lpmgpu_autotune, lpmgpu_set_cg_grid) on the device.

It times the persistent CG kernel on the problem's own matrix for several grid sizes, none above
the default, and keeps the fastest.  A tuned grid changes only the rounding of the CG's
reductions: load steps solved with it match those of the default grid within 1e-9 (FP64, Newton
counts equal) and 1e-7 (mixed), and every grid sets the candidates' per-iteration times."""
import numpy as np
import pytest

from _util import CFG, gpu_problem, rel

pytestmark = pytest.mark.gpu

TIGHT = dict(cg_rtol=1e-24, cg_atol=0.0)


def _steps(g, case, n):
    return _steps_from(g, case, 0, n)


def _steps_from(g, case, first, end):
    out = []
    for s in range(first, end):
        ok, st = g.solve_load_step(case.load_step(s))
        assert ok
        out.append((st["newton_solves"], g.state(("xyz",))["xyz"] - case.xyz))
    return out


@pytest.mark.parametrize("which,precision", [("hex", 0), ("sc", 0), ("hex", 1)])
def test_tuned_grid_solves_like_the_default(which, precision):
    case = (CFG.hex_plate(size=4.0, radius=0.1, steps=2, total_disp=0.002, tol_iter=1e-9) if which == "hex"
            else CFG.sc_cube(size=3.0, radius=0.2, steps=2, total_disp=0.002, tol_iter=1e-9))
    ref = gpu_problem(case, precision=precision, **TIGHT)
    base = _steps(ref, case, 2)
    ref.close()
    g = gpu_problem(case, precision=precision, **TIGHT)
    tuned = _steps(g, case, 1)  # the first step puts the displacement BCs in place
    res = g.autotune(iterations=30)
    assert res["precision"] == precision
    assert 1 <= len(res["candidates"]) <= 8 and res["candidates"][0] == res["grid_default"]
    assert all(1 <= c <= res["grid_default"] for c in res["candidates"])
    assert res["grid_chosen"] in res["candidates"]
    assert all(t > 0 for t in res["us_per_iter"])
    assert res["us_per_iter"][res["candidates"].index(res["grid_chosen"])] == min(res["us_per_iter"])
    # the tuner re-assembled K from the state after the first step and left that state as it was
    tuned += _steps_from(g, case, 1, 2)
    for (n0, u0), (n1, u1) in zip(base, tuned):
        if precision == 0:
            assert n0 == n1
        assert rel(u1, u0) <= (1e-9 if precision == 0 else 1e-7)
    g.close()


def test_set_cg_grid_forces_a_grid():
    """A forced small grid (down to one block) still solves the step; 0 restores the default."""
    case = CFG.hex_plate(size=3.0, radius=0.1, steps=1, total_disp=0.001, tol_iter=1e-9)
    ref = gpu_problem(case, **TIGHT)
    (n0, u0), = _steps(ref, case, 1)
    ref.close()
    for grid in (1, 3, 0):
        g = gpu_problem(case, **TIGHT)
        g.set_cg_grid(grid)
        (n1, u1), = _steps(g, case, 1)
        assert n1 == n0 and rel(u1, u0) <= 1e-9, grid
        g.close()
    with pytest.raises(Exception):
        g = gpu_problem(case, **TIGHT)
        try:
            g.set_cg_grid(-1)
        finally:
            g.close()
