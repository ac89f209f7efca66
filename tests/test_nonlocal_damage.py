"""Nonlocal damage on the device (through the C ABI) against the CPU oracle: elastic-damage
particles (include/particle_elastic_damage.h) whose local damage rates are averaged over the
neighbours that Assembly::searchNonlocalNeighbors finds (assembly.h:118-130, solver_static.h:32-62).

Bars: the same Newton solve counts per step (FP64), displacements within 1e-8 relative (FP64) and
1e-6 (mixed), damage within 1e-9 (FP64; the averaging's pow() weights may differ in the last bit
from the host's) and 1e-5 (mixed).  The oracle itself is pinned to the reference by the
hex_edamage golden fixture."""
import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, oracle_problem, oracle_step_args, rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,dtol,ktol", [(0, 1e-8, 1e-9), (1, 1e-6, 1e-5)])
def test_elastic_damage_matches_oracle(precision, dtol, ktol):
    case = CFG.edamage_plate()
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(case, precision=precision, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    for s in range(len(case.steps)):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg and oko
        if precision == 0:
            assert stg["newton_solves"] == sto["newton_solves"], f"step {s}"
        sg, so = g.state(), o.state()
        e = rel(sg["xyz"] - case.xyz, so["xyz"] - case.xyz)
        assert e <= dtol, f"step {s}: rel disp err {e}"
        dd = np.abs(sg["damage"] - so["damage"]).max()
        assert dd <= ktol, f"step {s}: damage differs by {dd}"
        assert rel(sg["state_var"], so["state_var"]) <= 100 * dtol
    assert so["damage"].max() > 0.5, "damage must grow over the load path"


def test_batch_elastic_damage_members_match_alone():
    """Two elastic-damage plates of different size in one batch: each as it is solved alone.
    Both sides solve tightly (at the reference's own CG tolerance these plates need 30 halvings
    in the oracle too); both load paths converge without a cut in the oracle."""
    cases = [CFG.edamage_plate(size=2.4), CFG.edamage_plate(size=2.0, total_disp=0.007)]
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    alone = []
    for c in cases:
        g = gpu_problem(c, **kw)
        stats = []
        for s in range(len(c.steps)):
            ok, st = g.solve_load_step(c.load_step(s))
            assert ok
            stats.append(st["newton_solves"])
        alone.append((g.state()["xyz"] - c.xyz, g.state()["damage"], stats))
        g.close()
    gs = [gpu_problem(c, **kw) for c in cases]
    b = LPM.Batch(0)
    mids = [b.add(g, [c.load_step(s) for s in range(len(c.steps))]) for g, c in zip(gs, cases)]
    b.run()
    for g, c, mid, (u0, d0, n0) in zip(gs, cases, mids, alone):
        info = b.member(mid)
        assert info["state"] == 1, info
        assert [st["newton_solves"] for st in b.member_steps(mid)] == n0
        st = g.state()
        assert rel(st["xyz"] - c.xyz, u0) <= 1e-8
        assert np.abs(st["damage"] - d0).max() <= 1e-9
    b.close()
    for g in gs:
        g.close()
