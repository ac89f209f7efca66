"""The bounded device-side waits of the persistent CG kernel.

Every grid-barrier wait of k_cg gives up after a time limit, records LPMGPU_ERR_TIMEOUT and lets
each block return, so a stuck barrier can never hang the GPU (the reference's MKL CG has no device
waits; its only failure report is a printout, solver.h:347-349).  The test shortens the limit to
1 ns on a problem whose CG runs hundreds of iterations over tens of blocks, so that some block's
natural barrier wait outlasts it, and expects the solve to fail with LPMGPU_ERR_TIMEOUT.  With the
default limit restored, the next solve on the same handle must match the CPU oracle's CG.  No
fault, trap or endless loop is involved: every wait is bounded by the limit it is given.
"""
import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, oracle_problem, oracle_step_args, rel

pytestmark = pytest.mark.gpu


def test_cg_barrier_timeout_is_reported_and_handle_recovers():
    # 10 x 10 mm hexagonal plate, 2,900 particles: about 90 slices, so about 90 blocks per barrier
    case = CFG.hex_plate(size=10.0, radius=0.1, steps=1, total_disp=0.001)
    g = gpu_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    g.apply_load_step(case.load_step(0))
    g.assemble(True)
    g.update_force_state()
    g.update_rr()
    r0 = g.residual().copy()

    g.set_wait_limit_ns(1)
    with pytest.raises(LPM.LpmGpuError) as ex:
        g.solve_linear()
    assert ex.value.status == LPM.ERR_TIMEOUT, str(ex.value)
    g.set_wait_limit_ns(0)  # back to the default

    # the handle is intact: same residual, and the next solve matches the oracle
    assert np.array_equal(g.residual(), r0)
    xg, st = g.solve_linear()
    assert st["cg_iters"] > 0
    o = oracle_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    o.update_geometry()
    o.update_force_state()
    o.apply_bc(*oracle_step_args(case, 0))
    o.assemble(True)
    o.update_geometry()
    o.update_force_state()
    o.update_rr()
    assert np.array_equal(g.residual(), o.residual())
    xo, _ = o.cg()
    assert rel(xg, xo) <= 1e-9, rel(xg, xo)

    # and a whole load step still converges on the handle
    ok, _ = g.solve_load_step(case.load_step(0))
    assert ok
    g.close()
