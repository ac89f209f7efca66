"""Serving loop (lpmgpu_server_*): solves submitted while others run give the results they give
alone.

Requests of different kinds (2D and 3D, elastic and J2, a pre-cracked plate, FP64 and mixed
precision) are submitted in two waves, the second while the first is on the GPU; the server
admits each against its HBM budget and runs it inside the shared batch.  Each result is compared
with the same problem solved alone through lpmgpu_solve_load_step, both sides with tight
tolerances (CG squared-norm test 1e-24 relative, Newton 1e-9): FP64 requests within 1e-8
relative displacement, mixed-precision ones within 1e-6 of the FP64 solution alone.
"""
import time

import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, rel

pytestmark = pytest.mark.gpu

TIGHT = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)


def _requests():
    return [
        (CFG.hex_plate(size=3.0, radius=0.1, steps=3, total_disp=0.003), 0),
        (CFG.sc_cube(size=2.4, radius=0.2, steps=3, total_disp=0.003), 0),
        (CFG.sc_cube(size=2.0, radius=0.25, steps=3, total_disp=0.06, ptype=LPM.ParticleType.J2Plasticity,
                     j2=(200.0, 0.0, 38714.0, 10.0)), 0),
        (CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=6, total_disp=0.006), 0),
        (CFG.hex_plate(size=4.0, radius=0.1, steps=4, total_disp=0.004), 1),
        (CFG.sc_cube(size=3.2, radius=0.2, steps=2, total_disp=0.002), 1),
    ]


def _alone(case):
    g = gpu_problem(case, **TIGHT)
    for s in range(len(case.steps)):
        ok, _ = g.solve_load_step(case.load_step(s))
        assert ok
    x = g.state(("xyz",))["xyz"]
    g.close()
    return x


def _submit(srv, case, precision):
    return srv.submit(case.assembly(), [case.load_step(s) for s in range(len(case.steps))],
                      undamaged_pt_type=case.undamaged_type, max_iter=case.max_iter, precision=LPM.Precision(precision),
                      **TIGHT)


@pytest.mark.parametrize("solo", [False, True])
def test_requests_submitted_while_others_run_match_alone(solo):
    """solo: every request solves its linear systems alone through the single-problem CG between
    the batched launches (lpmgpu_server_set_solo_bytes(1)), as the large requests of a stream do."""
    reqs = _requests()
    refs = [_alone(c) for c, _ in reqs]
    srv = LPM.Server()
    if solo:
        srv.set_solo_bytes(1)
    ids = [_submit(srv, c, p) for c, p in reqs[:3]]
    # the second wave arrives once the first is on the GPU
    t0 = time.time()
    while srv.stats()["running"] == 0 and srv.stats()["done"] < 3 and time.time() - t0 < 60:
        time.sleep(0.001)
    ids += [_submit(srv, c, p) for c, p in reqs[3:]]
    for (c, prec), rid, ref in zip(reqs, ids, refs):
        info = srv.wait(rid, timeout=300)
        assert info["state"] == 2, info
        assert info["steps_done"] == len(c.steps)
        x = srv.result(rid)
        tol = 1e-8 if prec == 0 else 1e-6
        e = rel(x - c.xyz, ref - c.xyz)
        assert e <= tol, f"{c.name} (precision {prec}): rel err {e}"
    st = srv.stats()
    assert st["done"] == len(reqs) and st["failed"] == 0 and st["worker_status"] == 0
    assert 0 <= st["latency_p50"] <= st["latency_p99"]
    srv.close()


def test_hbm_budget_bounds_resident_problems():
    """With a budget below one problem's admission estimate plus another one's real size, the
    requests are admitted one at a time: the memory held at once is one problem's, within the
    budget; all still complete."""
    cases = [CFG.sc_cube(size=3.2, radius=0.2, steps=2, total_disp=0.002) for _ in range(4)]
    ref = _alone(cases[0])
    probe = gpu_problem(cases[0])
    one = probe.sizes["device_bytes"]
    probe.close()
    est = LPM.Server.estimate_bytes(cases[0].assembly())
    assert est >= one
    budget = est + one // 2
    srv = LPM.Server(hbm_budget_bytes=budget)
    ids = [_submit(srv, c, 0) for c in cases]
    for c, rid in zip(cases, ids):
        info = srv.wait(rid, timeout=300)
        assert info["state"] == 2, info
        assert rel(srv.result(rid) - c.xyz, ref - c.xyz) <= 1e-8
    st = srv.stats()
    assert st["done"] == 4 and st["peak_bytes"] <= budget and st["peak_bytes"] < 2 * one, st
    srv.close()


def test_failed_request_reports_its_error():
    """A request whose problem cannot be built (a bond list naming a particle outside the
    problem) fails with a topology error instead of blocking the server."""
    c = CFG.hex_plate(size=2.0, radius=0.1, steps=1, total_disp=0.001)
    ass = c.assembly()
    nb0, nb1, p2 = CFG.bond_lists(c.xyz, LPM.UnitCell(c.lattice, c.radius))
    p2 = p2.copy()
    p2[0] = c.n + 5
    ass.bonds = (nb0, nb1, p2)
    srv = LPM.Server()
    rid = srv.submit(ass, [c.load_step(0)])
    good = _submit(srv, c, 0)
    info = srv.wait(rid, timeout=120)
    assert info["state"] == 3 and info["status"] == 7, info  # LPMGPU_ERR_TOPOLOGY
    with pytest.raises(LPM.LpmGpuError):
        srv.result(rid)
    assert srv.wait(good, timeout=120)["state"] == 2
    srv.close()
