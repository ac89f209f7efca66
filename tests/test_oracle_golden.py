"""Pins the CPU oracle (and the product's lattice generators) to the reference's own outputs.

The fixtures in tests/golden/ were produced by the LPM-CPP hot path compiled unmodified
(tests/golden/make_golden.py).  Topology, the reference CSR and the internal forces must be
bit-exact; positions after each load step agree to 1e-8 relative (the two CG loops sum the
sparse product in different orders: the reference's stand-in scatters the transposed half, and
at the reference's own CG tolerance that rounding difference reaches ~1e-10).
"""
import importlib
import json
import os

import numpy as np
import pytest

from _util import O, fatigue_cycles, fatigue_disp_scale, oracle_load_args, oracle_problem, oracle_step_args, rel

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

def _load_builders():
    import sys
    sys.path.insert(0, GOLDEN)
    mod = importlib.import_module("make_golden")
    return mod.cases()


CASES = _load_builders()
NAMES = sorted(CASES)
# cases run by SolverStatic; the fatigue cases run SolverFatigue's static steps and cycles
STATIC = [n for n in NAMES if not CASES[n][1].get("fatigue")]
FATIGUE = [n for n in NAMES if CASES[n][1].get("fatigue")]


def fixture(name):
    return np.load(os.path.join(GOLDEN, f"{name}.npz"))


@pytest.mark.parametrize("name", NAMES)
def test_generator_matches_reference(name):
    """The product's lattice generator reproduces the reference's particle ids and coordinates."""
    build, _ = CASES[name]
    case = build()
    g = fixture(name)
    assert np.array_equal(case.xyz, g["xyz0"])


@pytest.mark.parametrize("name", NAMES)
def test_oracle_topology_bit_exact(name):
    build, _ = CASES[name]
    case = build()
    g = fixture(name)
    o = oracle_problem(case)
    nb0, nb1, p2 = o.bonds()
    nconn, nlq, conns = o.conns()
    for k, v in (("nb0", nb0), ("nb1", nb1), ("bond_p2", p2), ("nconn", nconn), ("nlq", nlq), ("conns", conns)):
        assert np.array_equal(v, g[k]), k


@pytest.mark.parametrize("name", STATIC)
def test_oracle_load_steps(name):
    build, opts = CASES[name]
    case = build()
    g = fixture(name)
    kw = {}
    if "cg_tol" in opts:
        kw = dict(cg_rtol=opts["cg_tol"][0], cg_atol=opts["cg_tol"][1])
    tangent = bool(opts.get("tangent", False))
    o = oracle_problem(case, tangent=tangent, **kw)
    k_step = opts.get("dump_k", (0,))[-1]
    o.update_geometry()
    o.update_force_state()
    steps = g["steps"]
    for s in range(len(steps)):
        ok, st = o.solve_load_step(*oracle_step_args(case, s))
        assert ok
        if s == k_step and "K" in g.files:
            Kp, IK, JK, K = o.export_csr()
            assert np.array_equal(Kp, g["K_pointer"])
            assert np.array_equal(IK, g["IK"])
            assert np.array_equal(JK, g["JK"])
            if tangent or "damage_0" in g.files:
                # assembled from a solved (and, with continuous damage, damaged) state: carries
                # the CG's rounding
                assert np.abs(K - g["K"]).max() <= 1e-12 * np.abs(g["K"]).max()
            else:
                assert np.array_equal(K, g["K"]), "reference CSR values must be bit-exact"
        so = o.state()
        u_o = so["xyz"] - case.xyz
        u_r = g[f"xyz_{s}"] - g["xyz0"]
        assert rel(u_o, u_r) <= 1e-8, (s, rel(u_o, u_r))
        assert st["newton_solves"] == int(steps[s][0])
        assert st["cuts"] == int(steps[s][2])
        assert abs(st["cg_iters"] - int(steps[s][1])) <= max(3, 0.01 * steps[s][1])
        assert abs(st["reaction_norm"] - steps[s][3]) <= 1e-7 * steps[s][3]
        if f"state_var_{s}" in g.files:
            assert rel(so["state_var"], g[f"state_var_{s}"]) <= 1e-8
        if f"damage_{s}" in g.files:
            # the nonlocal rate is a weighted sum of pow() weights in the reference's order
            assert np.abs(so["damage"] - g[f"damage_{s}"]).max() <= 1e-10
        if f"bdamage_{s}" in g.files:
            if f"damage_{s}" in g.files:
                assert np.abs(so["bdamage"] - g[f"bdamage_{s}"]).max() <= 1e-10
            else:
                assert np.array_equal(so["bdamage"], g[f"bdamage_{s}"])


@pytest.mark.parametrize("name", FATIGUE)
def test_oracle_fatigue_cycles(name):
    """SolverFatigue (solver_fatigue.h): the static step of solveProblemStatic, then each cycle of
    solveProblemCyclic (generateLoadCycle, the dN/dt map, solveProblemOneCycle).  Per cycle: the
    same Newton solve count, the cycle count N, damage and the HCF state variables within 1e-12
    (bit-exact here; the nonlocal weights are pow() sums), the reaction history's norm within
    1e-12 relative.  Displacements are compared in absolute terms against the load amplitude:
    at a cycle's end the plate is unloaded and u is a residual of the CG's rounding."""
    build, opts = CASES[name]
    case = build()
    g = fixture(name)
    o = oracle_problem(case, cg_rtol=opts["cg_tol"][0], cg_atol=opts["cg_tol"][1])
    o.update_geometry()
    o.update_force_state()
    amp = fatigue_disp_scale(case)
    steps = g["steps"]
    results = []
    for s in range(len(case.steps)):
        ok, st = o.fatigue_static_step(*oracle_step_args(case, s))
        assert ok
        results.append(st)
    cyc = list(fatigue_cycles(case))
    assert len(case.steps) + len(cyc) == len(steps)
    for c, (N, dNdt, cycle) in enumerate(cyc):
        assert [N, dNdt] == list(g["cycles"][c])
        _, st = o.fatigue_cycle([oracle_load_args(x) for x in cycle], dNdt)
        results.append(st)
        s = len(case.steps) + c
        so = o.state()
        assert st["newton_solves"] == int(steps[s][0]), s
        assert np.abs(so["damage"] - g[f"damage_{s}"]).max() <= 1e-12, s
        assert np.abs(so["state_var"] - g[f"state_var_{s}"]).max() <= 1e-12 * np.abs(g[f"state_var_{s}"][:, 0]).max()
        assert np.abs(so["bdamage"] - g[f"bdamage_{s}"]).max() <= 1e-12, s
        du = np.abs((so["xyz"] - case.xyz) - (g[f"xyz_{s}"] - g["xyz0"])).max()
        assert du <= 1e-8 * amp, (s, du)
        assert abs(st["reaction_norm"] - steps[s][3]) <= 1e-12 * steps[s][3]
    assert g[f"damage_{len(steps) - 1}"].max() > 0.1, "damage must grow over the cycles"


def test_oracle_forces_bit_exact():
    """Internal forces of the undeformed hexagonal plate after the first load step's BCs."""
    build, _ = CASES["hex_small"]
    case = build()
    g = fixture("hex_small")
    o = oracle_problem(case)
    o.update_geometry()
    o.update_force_state()
    o.solve_load_step(*oracle_step_args(case, 0))
    assert rel(o.state()["pin"], g["pin_0"]) <= 1e-8


def test_fixture_meta_records_spec():
    for name in NAMES:
        meta = json.loads(str(fixture(name)["meta"]))
        assert meta["name"] == name and "lattice" in meta["spec"]


def test_planted_error_is_caught():
    """A perturbed stiffness entry in the oracle is detected by the bit-exact comparison."""
    build, _ = CASES["sc_small"]
    case = build()
    g = fixture("sc_small")
    o = oracle_problem(case)
    o.update_geometry()
    o.update_force_state()
    o.solve_load_step(*oracle_step_args(case, 0))
    K = o.export_csr()[3].copy()
    assert np.array_equal(K, g["K"])
    q = int(np.argmax(np.abs(K)))
    K[q] = np.nextafter(K[q], np.inf)
    assert not np.array_equal(K, g["K"])
