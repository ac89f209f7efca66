"""Batched solving (lpmgpu_batch_*): every member gives the result it gives alone.

Each case builds twin handles of the same problems.  One twin of each runs alone, load step by
load step, through lpmgpu_solve_load_step (the plain path); the others run together as members
of one batch, whose rounds send the pending Newton systems of each lane (a group of members with
its own share of the SMs) through one persistent CG launch.
The CG partition differs between the two (the batched kernel splits the GPU among the members),
so the two agree to rounding, not bit for bit.  Bars, with both sides solving tightly (CG
squared-norm test 1e-24 relative, Newton 1e-9):
  * FP64 members: per load step the same Newton solve count and cuts, the same broken bonds,
    displacements within 1e-8 relative of the member alone;
  * mixed-precision members: displacements within 1e-6 relative of the FP64 member alone;
  * members added while others are running give the same results as well.
"""
import numpy as np
import pytest

from _util import CFG, LPM, gpu_problem, hetero_plate, rel

pytestmark = pytest.mark.gpu

TIGHT = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
FP64_TOL = 1e-8
MIXED_TOL = 1e-6


def _cases():
    return [
        CFG.hex_plate(size=3.0, radius=0.1, steps=3, total_disp=0.003),
        CFG.sc_cube(size=2.4, radius=0.2, steps=3, total_disp=0.003),
        CFG.sc_cube(size=2.0, radius=0.25, steps=3, total_disp=0.06, ptype=LPM.ParticleType.J2Plasticity,
                    j2=(200.0, 0.0, 38714.0, 10.0)),
        CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=6, total_disp=0.006),
        hetero_plate(size=2.0, steps=2, total_disp=0.002),
    ]


def _cut_case():
    # a Newton cap of 5 makes the full step fail, so it is halved (solver_static.h:78-87)
    return CFG.hex_plate(size=2.0, radius=0.1, steps=1, total_disp=0.01)


def _alone(case, precision=0, max_iter=None):
    g = gpu_problem(case, precision=precision, max_iter=max_iter, **TIGHT)
    steps = []
    for s in range(len(case.steps)):
        ok, st = g.solve_load_step(case.load_step(s))
        assert ok
        steps.append(st)
    out = g.state()
    g.close()
    return out, steps


def _check_member(case, batch, mid, g, ref_state, ref_steps, tol, compare_counts=True):
    info = batch.member(mid)
    assert info["state"] == 1 and info["status"] == 0, info
    assert info["steps_done"] == len(case.steps)
    steps = batch.member_steps(mid)
    if compare_counts:
        for s, (a, b) in enumerate(zip(steps, ref_steps)):
            assert a["newton_solves"] == b["newton_solves"], (case.name, s, a, b)
            assert a["cuts"] == b["cuts"], (case.name, s)
    st = g.state()
    e = rel(st["xyz"] - case.xyz, ref_state["xyz"] - case.xyz)
    assert e <= tol, f"{case.name}: displacement rel err {e}"
    if compare_counts:
        assert np.array_equal(st["bdamage"] == 1.0, ref_state["bdamage"] == 1.0), case.name
    return info


@pytest.mark.parametrize("lanes", [1, 3])
def test_batch_fp64_members_match_alone(lanes):
    """With one lane every round launches all members' CGs together; with three, the members are
    dealt to three lanes whose launches run side by side on shares of the SMs."""
    cases = _cases() + [_cut_case()]
    max_iters = [None] * (len(cases) - 1) + [5]
    refs = [_alone(c, max_iter=mi) for c, mi in zip(cases, max_iters)]
    batch = LPM.Batch()
    batch.set_lanes(lanes)
    gs, mids = [], []
    for c, mi in zip(cases, max_iters):
        g = gpu_problem(c, max_iter=mi, **TIGHT)
        gs.append(g)
        mids.append(batch.add(g, [c.load_step(s) for s in range(len(c.steps))]))
    batch.run()
    for c, g, mid, (ref_state, ref_steps) in zip(cases, gs, mids, refs):
        _check_member(c, batch, mid, g, ref_state, ref_steps, FP64_TOL)
    assert batch.member_steps(mids[-1])[0]["cuts"] > 0
    st = batch.stats()
    assert st["members_done"] == len(cases) and st["members_failed"] == 0
    assert st["cg_launches"] > 0 and st["dof_iters"] > 0
    batch.close()
    for g in gs:
        g.close()


@pytest.mark.parametrize("lanes,kernel", [(1, None), (2, None), (1, "0"), (1, "1"), (1, "2"), (1, "3")])
def test_batch_mixed_members_match_fp64_alone(lanes, kernel, monkeypatch):
    """Mixed members (FP32 inner solves in FP64 refinement) against FP64 alone, with the batch's
    own choice of the FP32 kernel (kernel None: its tuner tries the four over the first launches)
    and with each kernel fixed: 0 the two-reduction CG, 1 and 2 the single-reduction CG with one or
    two SpMV steps in flight, 3 the single-reduction CG whose SpMV reads the matrix from shared
    memory, streamed there by bulk asynchronous copies."""
    if kernel is not None:
        monkeypatch.setenv("LPMGPU_BATCH_SR", kernel)
    else:
        monkeypatch.delenv("LPMGPU_BATCH_SR", raising=False)
    cases = _cases()[:3]
    refs = [_alone(c) for c in cases]
    batch = LPM.Batch()
    batch.set_lanes(lanes)
    gs, mids = [], []
    for c in cases:
        g = gpu_problem(c, precision=1, **TIGHT)
        gs.append(g)
        mids.append(batch.add(g, [c.load_step(s) for s in range(len(c.steps))]))
    batch.run()
    for c, g, mid, (ref_state, ref_steps) in zip(cases, gs, mids, refs):
        info = _check_member(c, batch, mid, g, ref_state, ref_steps, MIXED_TOL, compare_counts=False)
        assert info["total"]["refinements"] > 0
    st = batch.stats()
    assert st["fp32_kernel"] in (0, 1, 2, 3)
    assert st["fp32_kernel_small"] in (0, 1, 2, 3)
    if kernel is not None:
        assert st["fp32_kernel"] == st["fp32_kernel_small"] == int(kernel) and st["fp32_tuning"] == 0
    batch.close()
    for g in gs:
        g.close()


@pytest.mark.parametrize("lanes", [1, 2])
def test_batch_members_join_while_others_run(lanes):
    """Continuous batching: members added between rounds, while earlier members are mid-path
    (with two lanes, also while the other lane's launch is in flight)."""
    cases = _cases()
    refs = [_alone(c) for c in cases]
    batch = LPM.Batch()
    batch.set_lanes(lanes)
    gs = [gpu_problem(c, **TIGHT) for c in cases]
    mids = [None] * len(cases)
    mids[0] = batch.add(gs[0], [cases[0].load_step(s) for s in range(len(cases[0].steps))])
    nxt, rounds = 1, 0
    running = 1
    while running > 0 or nxt < len(cases):
        if nxt < len(cases) and rounds % 3 == 2:
            mids[nxt] = batch.add(gs[nxt], [cases[nxt].load_step(s) for s in range(len(cases[nxt].steps))])
            nxt += 1
        running = batch.round()
        rounds += 1
        assert rounds < 100000
    for c, g, mid, (ref_state, ref_steps) in zip(cases, gs, mids, refs):
        _check_member(c, batch, mid, g, ref_state, ref_steps, FP64_TOL)
        batch.remove(mid)
    batch.close()
    for g in gs:
        g.close()


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, MIXED_TOL)])
def test_batch_paused_solves_resume(precision, tol, monkeypatch):
    """A launch runs at most `slice` CG iterations; unfinished solves pause and resume in the
    next round with their Krylov state.  A 7-iteration slice makes every solve pause many
    times; the results still match the members alone.  Mixed members: the batch's tuner cycles
    the FP32 kernels over its first launches, so paused inner solves meet kernels of the other
    family (whose Krylov state differs); such a solve ends its inner solve and restarts from the
    true residual, so no inner solve runs to its cap and the members' CG iterations stay within
    twice those of the mixed solves alone."""
    monkeypatch.delenv("LPMGPU_BATCH_SR", raising=False)
    cases = _cases()[:4]
    refs = [_alone(c) for c in cases]
    mixed_iters = [sum(st["cg_iters"] for st in _alone(c, precision=1)[1]) for c in cases] if precision else None
    batch = LPM.Batch()
    batch.set_slice(7)
    gs, mids = [], []
    for c in cases:
        g = gpu_problem(c, precision=precision, **TIGHT)
        gs.append(g)
        mids.append(batch.add(g, [c.load_step(s) for s in range(len(c.steps))]))
    batch.run()
    for k, (c, g, mid, (ref_state, ref_steps)) in enumerate(zip(cases, gs, mids, refs)):
        info = _check_member(c, batch, mid, g, ref_state, ref_steps, tol, compare_counts=(precision == 0))
        if precision:
            assert info["total"]["cg_maxit_hits"] == 0, (c.name, info["total"])
            assert info["total"]["cg_iters"] <= 2 * mixed_iters[k], (c.name, info["total"]["cg_iters"], mixed_iters[k])
    assert batch.stats()["cg_launches"] > 20
    batch.close()
    for g in gs:
        g.close()


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, MIXED_TOL)])
def test_batch_solo_members_match_alone(precision, tol):
    """Solo members (lpmgpu_batch_set_solo_bytes: those whose CG streams at least that many bytes
    per iteration) solve their linear systems alone through the single-problem CG between the
    batched launches, while the other members share the launches.  Every member matches its twin
    alone in the same precision; an FP64 solo member takes exactly the alone path's steps, so it
    matches bit for bit."""
    cases = _cases()
    refs = [_alone(c, precision=precision) for c in cases]
    batch = LPM.Batch()
    gs, mids = [], []
    for k, c in enumerate(cases):
        batch.set_solo_bytes(1 if k % 2 == 0 else 0)  # members 0, 2, 4 solo
        g = gpu_problem(c, precision=precision, **TIGHT)
        gs.append(g)
        mids.append(batch.add(g, [c.load_step(s) for s in range(len(c.steps))]))
    batch.run()
    for k, (c, g, mid, (ref_state, ref_steps)) in enumerate(zip(cases, gs, mids, refs)):
        _check_member(c, batch, mid, g, ref_state, ref_steps, tol, compare_counts=(precision == 0))
        if precision == 0 and k % 2 == 0:
            assert np.array_equal(g.state()["xyz"], ref_state["xyz"]), c.name
    st = batch.stats()
    assert st["solo_solves"] > 0 and st["cg_launches"] > 0
    batch.close()
    for g in gs:
        g.close()


@pytest.mark.parametrize("precision,tol", [(0, FP64_TOL), (1, MIXED_TOL)])
def test_batch_tangent_members_match_alone(precision, tol):
    """Tangent-mode members (K re-assembled before every Newton solve) in a batch give the
    results they give alone."""
    cases = [CFG.fcc_bar(size=(1.6, 1.6, 2.4), radius=0.2, steps=3, strain=0.02),
             CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=6, total_disp=0.006)]
    refs = []
    for c in cases:
        g = gpu_problem(c, tangent=True, **TIGHT)
        st = []
        for s in range(len(c.steps)):
            ok, x = g.solve_load_step(c.load_step(s))
            assert ok
            st.append(x)
        refs.append((g.state(), st))
        g.close()
    batch = LPM.Batch()
    gs, mids = [], []
    for c in cases:
        g = gpu_problem(c, precision=precision, tangent=True, **TIGHT)
        gs.append(g)
        mids.append(batch.add(g, [c.load_step(s) for s in range(len(c.steps))]))
    batch.run()
    for c, g, mid, (ref_state, ref_steps) in zip(cases, gs, mids, refs):
        _check_member(c, batch, mid, g, ref_state, ref_steps, tol, compare_counts=(precision == 0))
    batch.close()
    for g in gs:
        g.close()
