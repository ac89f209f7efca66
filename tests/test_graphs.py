"""The force-state sequence of every Newton iteration (geometry and bond forces, particle forces
and the residual, the scalar record's copy) and the state store / reset copies are replayed from
CUDA graphs captured when the problem is created.
The graph holds the same kernels with the same arguments as the direct launches, so a load path
solved with it is bit-identical to one solved with LPMGPU_NO_GRAPHS set, with the same kernel
count."""
import os

import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem

pytestmark = pytest.mark.gpu


def _run(case, graphs):
    old = os.environ.pop("LPMGPU_NO_GRAPHS", None)
    if not graphs:
        os.environ["LPMGPU_NO_GRAPHS"] = "1"
    try:
        g = gpu_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    finally:
        os.environ.pop("LPMGPU_NO_GRAPHS", None)
        if old is not None:
            os.environ["LPMGPU_NO_GRAPHS"] = old
    out = []
    for s in range(len(case.steps)):
        ok, st = g.solve_load_step(case.load_step(s))
        assert ok
        out.append((st["newton_solves"], st["cg_iters"], g.state(("xyz", "damage", "bdamage"))))
    launches = g.counters()["kernel_launches"]
    g.close()
    return out, launches


@pytest.mark.parametrize("which", ["hex_damage", "sc_j2"])
def test_graph_replay_is_bit_identical_to_direct_launches(which):
    if which == "hex_damage":
        case = CFG.hex_plate(size=2.0, radius=0.1, steps=3, total_disp=0.024, critical_bstrain=3e-3, tol_iter=1e-9)
    else:
        case = CFG.sc_cube(size=2.0, radius=0.25, steps=3, total_disp=0.06, tol_iter=1e-9,
                           ptype=LPM.ParticleType.J2Plasticity, j2=(200.0, 0.0, 38714.0, 10.0))
    a, la = _run(case, True)
    b, lb = _run(case, False)
    assert la == lb
    for (na, ia, sa), (nb, ib, sb) in zip(a, b):
        assert (na, ia) == (nb, ib)
        for k in sa:
            assert np.array_equal(sa[k], sb[k], equal_nan=True), k  # J2 damage is NaN without a nonlocal search
