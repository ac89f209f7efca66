"""Further device parity cases, through the C ABI against the CPU oracle: the known-answer beam
of examples/ex7_convergence_beam.cpp, whose load is a force BC (Solver::updateForceBC,
solver.h:167-188); elastic-damage particles with undamaged grips (the undamaged type in
SolverStatic::updateStaticDamage, solver_static.h:32-62); and an FCC cube with cubic elastic
constants (setParticleProperty's (C11, C12, C44) overload, particle_elastic.h:110-140, as
examples/ex3_singlecrystal_3d_fcc.cpp sets them).  The oracles are pinned to the reference: the
beam by its known answer (tests/test_beam_kat.py), the others by the hex_edamage_grips and
fcc_cubic golden fixtures."""
import numpy as np
import pytest

from _util import CFG, gpu_problem, oracle_problem, oracle_step_args, rel
from test_beam_kat import BEAM_L2_REFERENCE, beam_l2_error

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(0, 1e-8), (1, 1e-6)])
def test_device_beam_force_bc_known_answer(precision, tol):
    """The beam through the C ABI: its load is a force BC, shared by the left edge's particles
    (Solver::updateForceBC, solver.h:167-188, the device's k_force_bc).  Solved tightly on both
    sides, the device's displacements match the oracle's within 1e-8 (FP64) or 1e-6 (mixed);
    at the example's own tolerances the device's L2 error is the known answer within 1e-6.
    "Tightly" is Newton 1e-7: below about 1e-8 the beam's residual stops falling (rounding of the
    force sums), Newton fails, and the halved retry keeps the failed attempt's external force (the
    reference's resetStateVar leaves Pex alone), which doubles the load."""
    from _util import gpu_problem
    case = CFG.cantilever_beam()
    m = case.meta
    args = (m["length"], m["depth"], m["force"], case.material.E, case.material.mu)
    tight = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-7)
    o = oracle_problem(case, **tight)
    o.update_geometry()
    o.update_force_state()
    ok, st = o.solve_load_step(*oracle_step_args(case, 0))
    assert ok and st["cuts"] == 0
    x_o = o.state()["xyz"]
    g = gpu_problem(case, precision=precision, **tight)
    ok, st = g.solve_load_step(case.load_step(0))
    assert ok and st["cuts"] == 0
    x_g = g.state()["xyz"]
    g.close()
    assert rel(x_g - case.xyz, x_o - case.xyz) <= tol
    if precision == 0:
        g = gpu_problem(case)
        ok, st = g.solve_load_step(case.load_step(0))
        assert ok and st["newton_solves"] == 2
        e = beam_l2_error(case.xyz, g.state()["xyz"], *args)
        g.close()
        assert abs(e - BEAM_L2_REFERENCE) <= 1e-6 * BEAM_L2_REFERENCE


def test_elastic_damage_with_undamaged_grips_matches_oracle():
    """Type-3 grips near the top and bottom edges as the undamaged type: they take no damage and
    are left out of the averaging (solver_static.h:37-57); FP64 bars as above.  The oracle is
    pinned to the reference by the hex_edamage_grips golden fixture."""
    case = CFG.edamage_plate(undamaged_band=0.5)
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(case, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    grips = case.types == 3
    assert grips.any()
    for s in range(len(case.steps)):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg and oko
        assert stg["newton_solves"] == sto["newton_solves"], f"step {s}"
        sg, so = g.state(), o.state()
        assert rel(sg["xyz"] - case.xyz, so["xyz"] - case.xyz) <= 1e-8, f"step {s}"
        assert np.abs(sg["damage"] - so["damage"]).max() <= 1e-9, f"step {s}"
        assert (sg["damage"][grips] == 0).all()
    g.close()



def test_cubic_constants_fcc_matches_oracle():
    """Topology and the reference CSR pattern bit-exact, the stiffness before the BC elimination
    bit-exact from the exact kernel and within 1e-12 from the fast one, and the load steps' Newton
    counts equal with displacements within 1e-8."""
    case = CFG.fcc_cubic_cube(steps=3, total_disp=0.003)
    tight = dict(cg_rtol=1e-24, cg_atol=0.0)
    g = gpu_problem(case, **tight)
    o = oracle_problem(case, **tight)
    t = g.topology()
    nb0, nb1, p2 = o.bonds()
    nconn, nlq, conns = o.conns()
    for k, v in (("nb0", nb0), ("nb1", nb1), ("bond_p2", p2), ("nconn", nconn), ("nlq", nlq), ("conns", conns)):
        assert np.array_equal(t[k], v), k
    o.update_geometry()
    o.update_force_state()
    o.assemble(False)
    ref = o.export_csr()
    # the bit-exact kernel: every array equal; the fast form (the default): values within 1e-12
    g.set_assembly_exact(True)
    g.assemble(False)
    for a, b in zip(g.export_csr(), ref):
        assert np.array_equal(a, b)
    g.set_assembly_exact(False)
    g.assemble(False)
    K = g.export_csr()[3]
    assert np.abs(K - ref[3]).max() <= 1e-12 * np.abs(ref[3]).max()
    for s in range(len(case.steps)):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg and oko
        assert stg["newton_solves"] == sto["newton_solves"], s
        assert rel(g.state(("xyz",))["xyz"] - case.xyz, o.state()["xyz"] - case.xyz) <= 1e-8, s
    g.close()
