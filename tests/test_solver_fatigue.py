"""SolverFatigue on the device (include/solver_fatigue.h, include/particle_fatigue_hcf.h), through
the C ABI, against the CPU oracle.  The oracle is pinned to the reference's own SolverFatigue by
the hex_fatigue golden fixture.

The case: a hexagonal plate of fatigue HCF particles, one static step of solveProblemStatic, then
constant-amplitude displacement cycles of solveProblemCyclic; damage grows every cycle and
reaches 1 at two particles in the last one.

Bars, per cycle: FP64 — the same Newton solve count, damage within 1e-9 (the nonlocal weights and
the rate law use the device's pow(), which may differ from the host's in the last bit), the HCF
state variables within 1e-9 relative, displacements within 1e-8 x the load amplitude (at a cycle's
end the plate is unloaded, so u is compared in absolute terms); mixed precision — damage within
1e-5, displacements within 1e-6 x the amplitude."""
import numpy as np
import pytest

from _util import CFG, LPM, fatigue_cycles, fatigue_disp_scale, gpu_problem, oracle_load_args, oracle_problem, oracle_step_args

pytestmark = pytest.mark.gpu

TIGHT = dict(cg_rtol=1e-24, cg_atol=0.0)


def _oracle_run(case):
    o = oracle_problem(case, **TIGHT)
    o.update_geometry()
    o.update_force_state()
    out = []
    for s in range(len(case.steps)):
        ok, st = o.fatigue_static_step(*oracle_step_args(case, s))
        assert ok
        out.append((st, o.state()))
    for N, dNdt, steps in fatigue_cycles(case):
        _, st = o.fatigue_cycle([oracle_load_args(x) for x in steps], dNdt)
        out.append((st, o.state()))
    return out


@pytest.mark.parametrize("load,precision,dtol,ktol", [("disp", 0, 1e-8, 1e-9), ("disp", 1, 1e-6, 1e-5),
                                                      ("force", 0, 1e-8, 1e-9), ("dogbone3d", 0, 1e-8, 1e-9),
                                                      ("ct", 0, 1e-8, 1e-9), ("grips", 0, 1e-8, 1e-9)])
def test_fatigue_cycles_match_oracle(load, precision, dtol, ktol):
    case = {"disp": lambda: CFG.fatigue_plate(),
            "force": lambda: CFG.fatigue_plate(load_type="uniaxial_force", amplitude=200.0, cycles=4, tol_iter=1e-7),
            "dogbone3d": lambda: CFG.fatigue_cube(),
            "ct": lambda: CFG.fatigue_plate(load_type="ct_force", amplitude=250.0, cycles=4, tol_iter=1e-7),
            "grips": lambda: CFG.fatigue_plate(undamaged_band=0.5)}[load]()
    amp = fatigue_disp_scale(case)
    ref = _oracle_run(case)
    g = gpu_problem(case, precision=precision, **TIGHT)
    got = []
    for s in range(len(case.steps)):
        ok, st = g.fatigue_static_step(case.load_step(s))
        assert ok
        got.append((st, g.state()))
    for N, dNdt, steps in fatigue_cycles(case):
        _, st = g.fatigue_cycle(steps, dNdt)
        assert st["converged"]
        got.append((st, g.state()))
    assert len(got) == len(ref)
    for k, ((sg, xg), (so, xo)) in enumerate(zip(got, ref)):
        if precision == 0:
            assert sg["newton_solves"] == so["newton_solves"], k
        du = np.abs((xg["xyz"] - case.xyz) - (xo["xyz"] - case.xyz)).max()
        assert du <= dtol * amp, (k, du)
        dd = np.abs(xg["damage"] - xo["damage"]).max()
        assert dd <= ktol, (k, dd)
        assert np.abs(xg["bdamage"] - xo["bdamage"]).max() <= ktol, k
        sv_scale = max(np.abs(xo["state_var"][:, 0]).max(), 1e-300)
        assert np.abs(xg["state_var"][:, [0, 2]] - xo["state_var"][:, [0, 2]]).max() <= 100 * ktol * sv_scale, k
    assert ref[-1][1]["damage"].max() > (0.99 if load == "disp" else 0.1), "damage must grow over the cycles"


def test_solver_fatigue_mirror_runs_the_cyclic_loop(tmp_path):
    """The Python mirror of SolverFatigue (readLoad, solveProblemStatic, solveProblemCyclic) gives
    the oracle's final state, and its dump file holds one frame per static step and per cycle."""
    case = CFG.fatigue_plate()
    fat = case.meta["fatigue"]
    amp = max(abs(v) for v in fat["spectrum"])
    ref = _oracle_run(case)
    spec = tmp_path / "load.txt"
    spec.write_text("\n".join(repr(v) for v in fat["spectrum"]) + "\n")
    dump = tmp_path / "fatigue.dump"
    solv = LPM.SolverFatigue(case.undamaged_type, case.assembly(), LPM.StiffnessMode.Analytical, LPM.SolverMode.CG,
                             LPM.TimeMapMode.Linear, fat["tau"], str(dump), case.max_iter, case.tol_iter, **TIGHT)
    start = solv.solveProblemStatic([case.load_step(s) for s in range(len(case.steps))], 0)
    assert start == len(case.steps)
    solv.readLoad(str(spec))
    N = solv.solveProblemCyclic(LPM.FatigueLoadType.LoadUniaxialDisp, fat["n_interval"],
                                [case.groups[g] for g in fat["groups"]])
    assert N == int(0.5 * (len(fat["spectrum"]) - 1))
    st = solv.problem.state()
    xo = ref[-1][1]
    assert np.abs((st["xyz"] - case.xyz) - (xo["xyz"] - case.xyz)).max() <= 1e-8 * amp
    assert np.abs(st["damage"] - xo["damage"]).max() <= 1e-9
    frames = dump.read_text().count("ITEM: TIMESTEP")
    assert frames == len(ref)
    solv.problem.close()


def test_fatigue_update_damage_alone_matches_oracle():
    """updateFatigueDamage on its own after the static step and one loading step: the nonlocal
    average and the rate x dN/dt update, and the cleared cycle extremes."""
    case = CFG.fatigue_plate()
    o = oracle_problem(case, **TIGHT)
    o.update_geometry()
    o.update_force_state()
    g = gpu_problem(case, **TIGHT)
    o.fatigue_static_step(*oracle_step_args(case, 0))
    g.fatigue_static_step(case.load_step(0))
    _, _, steps = next(iter(fatigue_cycles(case)))
    o.fatigue_cycle([oracle_load_args(steps[0])], 0.0)
    g.fatigue_cycle([steps[0]], 0.0)
    for dNdt in (3.0, 5.0):
        ao = o.fatigue_update_damage(dNdt)
        ag = g.fatigue_update_damage(dNdt)
        assert ao == ag
        so, sg = o.state(), g.state()
        assert np.abs(sg["damage"] - so["damage"]).max() <= 1e-9
        assert np.array_equal(sg["state_var"][:, 1:], so["state_var"][:, 1:])
    g.close()


def _run_both(case, tmp_path):
    import os
    from _util import O
    for b in (O.REF_BIN, O.REF_GPU_BIN):
        if not os.path.exists(b):
            pytest.skip(f"{os.path.basename(b)} not built (make -C oracle ref ref-gpu)")
    out = {}
    for tag, binary in (("cpu", O.REF_BIN), ("gpu", O.REF_GPU_BIN)):
        d = str(tmp_path / tag)
        spec = O.write_ref_spec(case, d, cg_tol=(1e-24, 0.0), loop="ref")
        O.run_ref(spec, d, threads=1, timeout=900, binary=binary)
        out[tag] = d
    return out


def test_solver_fatigue_gpu_cpp_matches_solver_fatigue(tmp_path):
    """The C++ drop-in SolverFatigueGPU (lpm-cpp_b200/cpp/solver_static_gpu.h) against the
    reference's SolverFatigue: the same driver (oracle/ref_driver.cpp) built both ways, the
    reference's Assembly, fatigue particles (with their nonlocal lists) and LoadStep templates
    feeding the device library.  Per static step and cycle: Newton solves equal, damage within
    1e-9, displacements within 1e-8 x the amplitude, the same cycle counts."""
    from _util import O
    case = CFG.fatigue_plate()
    amp = max(abs(v) for v in case.meta["fatigue"]["spectrum"])
    out = _run_both(case, tmp_path)
    rc, rg = O.read_ref_steps(out["cpu"]), O.read_ref_steps(out["gpu"])
    assert len(rc) == len(rg) == 5
    with open(f"{out['cpu']}/cycles.txt") as a, open(f"{out['gpu']}/cycles.txt") as b:
        assert a.read() == b.read()
    x0 = O.read_bin(out["cpu"], "xyz0.f64", np.float64)
    for s in range(len(rc)):
        assert rc[s]["newton_solves"] == rg[s]["newton_solves"], s
        t = f"{s:03d}"
        uc = O.read_bin(out["cpu"], f"xyz_{t}.f64", np.float64) - x0
        ug = O.read_bin(out["gpu"], f"xyz_{t}.f64", np.float64) - x0
        assert np.abs(ug - uc).max() <= 1e-8 * amp, s
        dc = O.read_bin(out["cpu"], f"damage_{t}.f64", np.float64)
        dg = O.read_bin(out["gpu"], f"damage_{t}.f64", np.float64)
        assert np.abs(dg - dc).max() <= 1e-9, s
    assert dc.max() >= 1.0


def test_solver_static_gpu_passes_the_assembly_nonlocal_lists(tmp_path):
    """SolverStaticGPU with elastic-damage particles on which the example ran
    searchNonlocalNeighbors: the adapter hands the Assembly's own nonlocal lists to the device
    (lpmgpu_desc.nonlocal_count / nonlocal_ids), and the nonlocal damage follows SolverStatic."""
    from _util import O, rel
    case = CFG.edamage_plate()
    out = _run_both(case, tmp_path)
    rc, rg = O.read_ref_steps(out["cpu"]), O.read_ref_steps(out["gpu"])
    assert len(rc) == len(rg) == len(case.steps)
    x0 = O.read_bin(out["cpu"], "xyz0.f64", np.float64)
    for s in range(len(rc)):
        assert rc[s]["newton_solves"] == rg[s]["newton_solves"], s
        t = f"{s:03d}"
        uc = O.read_bin(out["cpu"], f"xyz_{t}.f64", np.float64) - x0
        ug = O.read_bin(out["gpu"], f"xyz_{t}.f64", np.float64) - x0
        assert rel(ug, uc) <= 1e-8, s
        dc = O.read_bin(out["cpu"], f"damage_{t}.f64", np.float64)
        dg = O.read_bin(out["gpu"], f"damage_{t}.f64", np.float64)
        assert np.abs(dg - dc).max() <= 1e-9, s
    assert dc.max() > 0.5


def test_batch_fatigue_members_match_alone():
    """Two fatigue plates (displacement- and force-driven) as fatigue members of one batch
    (lpmgpu_batch_add_fatigue), their Newton systems solved by the batched CG with the other
    member's: each ends as it does alone through lpmgpu_fatigue_static_step / _cycle (damage
    within 1e-9, displacements within 1e-8 x the scale, the same Newton count)."""
    cases = [CFG.fatigue_plate(),
             CFG.fatigue_plate(size=2.0, load_type="uniaxial_force", amplitude=200.0, cycles=4, tol_iter=1e-7)]
    alone = []
    for c in cases:
        g = gpu_problem(c, **TIGHT)
        newton = 0
        for s in range(len(c.steps)):
            ok, st = g.fatigue_static_step(c.load_step(s))
            assert ok
            newton += st["newton_solves"]
        for N, dNdt, steps in fatigue_cycles(c):
            _, st = g.fatigue_cycle(steps, dNdt)
            newton += st["newton_solves"]
        alone.append((g.state(("xyz", "damage")), newton))
        g.close()
    gs = [gpu_problem(c, **TIGHT) for c in cases]
    b = LPM.Batch(0)
    mids = []
    for g, c in zip(gs, cases):
        cyc = list(fatigue_cycles(c))
        mids.append(b.add_fatigue(g, [c.load_step(s) for s in range(len(c.steps))], [x[2] for x in cyc],
                                  [x[1] for x in cyc]))
    b.run()
    for g, c, mid, (st0, n0) in zip(gs, cases, mids, alone):
        info = b.member(mid)
        assert info["state"] == 1, info
        assert sum(s["newton_solves"] for s in b.member_steps(mid)) == n0
        st = g.state(("xyz", "damage"))
        scale = fatigue_disp_scale(c)
        assert np.abs((st["xyz"] - c.xyz) - (st0["xyz"] - c.xyz)).max() <= 1e-8 * scale
        assert np.abs(st["damage"] - st0["damage"]).max() <= 1e-9
    assert max(alone[0][0]["damage"].max(), alone[1][0]["damage"].max()) > 0.1
    b.close()
    for g in gs:
        g.close()


def test_served_fatigue_request_matches_alone():
    """A fatigue run submitted to the server (lpmgpu_server_submit_fatigue) while a static
    request runs: its final positions are those of the same run alone within 1e-8 x the scale."""
    c = CFG.fatigue_plate()
    g = gpu_problem(c, **TIGHT)
    for s in range(len(c.steps)):
        g.fatigue_static_step(c.load_step(s))
    cyc = list(fatigue_cycles(c))
    for N, dNdt, steps in cyc:
        g.fatigue_cycle(steps, dNdt)
    x_alone = g.state(("xyz",))["xyz"]
    g.close()
    other = CFG.hex_plate(size=3.0, radius=0.1, steps=3, total_disp=0.003, tol_iter=1e-9)
    srv = LPM.Server(0, hbm_budget_bytes=8 * 10**9)
    r0 = srv.submit(other.assembly(), [other.load_step(s) for s in range(3)], tol_iter=other.tol_iter, **TIGHT)
    r1 = srv.submit_fatigue(c.assembly(), [c.load_step(s) for s in range(len(c.steps))], [x[2] for x in cyc],
                            [x[1] for x in cyc], undamaged_pt_type=c.undamaged_type, max_iter=c.max_iter,
                            tol_iter=c.tol_iter, **TIGHT)
    for rid in (r0, r1):
        info = srv.wait(rid, timeout=300)
        assert info["state"] == 2, info
    x = srv.result(r1).reshape(-1, 3)
    assert np.abs((x - c.xyz) - (x_alone - c.xyz)).max() <= 1e-8 * fatigue_disp_scale(c)
    srv.close()


def test_grid_nonlocal_search_gives_the_all_pairs_run():
    """The nonlocal search by cell grid (the default above 16,384 particles) and by all pairs
    (LPMGPU_NL_GRID forces either) give the same lists in the same order, so a fatigue run is
    bit-identical with either."""
    import os
    c = CFG.fatigue_plate()
    states = []
    for mode in ("1", "0"):
        os.environ["LPMGPU_NL_GRID"] = mode
        try:
            g = gpu_problem(c, **TIGHT)
        finally:
            os.environ.pop("LPMGPU_NL_GRID", None)
        g.fatigue_static_step(c.load_step(0))
        for N, dNdt, steps in fatigue_cycles(c):
            g.fatigue_cycle(steps, dNdt)
        states.append(g.state(("xyz", "damage", "state_var")))
        g.close()
    for k in states[0]:
        assert np.array_equal(states[0][k], states[1][k]), k


def test_device_nonlocal_lists_at_scale():
    """The nonlocal lists of a 26 mm plate (19,500 particles: the cell-grid search) read back from
    the device (lpmgpu_get_nonlocal) equal the all-pairs lists, both the device's own
    (LPMGPU_NL_GRID=0) and numpy's: every particle within cutoff_ratio x nonlocal_L, by
    Particle::distanceTo's arithmetic, in ascending id."""
    import os
    from scipy.spatial import cKDTree
    c = CFG.fatigue_plate(size=26.0)
    assert c.n > 16384
    rc = c.nonlocal_cutoff_ratio * c.material.nonlocal_L
    lists = []
    for mode in (None, "0"):
        if mode is not None:
            os.environ["LPMGPU_NL_GRID"] = mode
        try:
            g = gpu_problem(c)
        finally:
            os.environ.pop("LPMGPU_NL_GRID", None)
        lists.append(g.nonlocal_lists())
        g.close()
    (cg, ig), (ca, ia) = lists
    assert np.array_equal(cg, ca) and np.array_equal(ig, ia)
    x = c.xyz
    cand = cKDTree(x).query_ball_point(x, rc * (1 + 1e-9))
    start = np.concatenate([[0], np.cumsum(cg)])
    for i in range(c.n):
        js = np.array(sorted(cand[i]), dtype=np.int64)
        d = x[i] - x[js]
        dist = np.sqrt(d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        want = js[dist < rc]
        assert np.array_equal(ig[start[i]:start[i + 1]], want), i
