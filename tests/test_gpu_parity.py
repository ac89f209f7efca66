"""Parity of the device path (through the C ABI) with the CPU oracle on the same inputs.

Bars: bond lists, connection lists and the reference CSR pattern bit-exact; internal forces
bit-exact; stiffness entries within 1e-12 of max|K| (bit-exact except the BC diagonal, whose
norm is a tree sum on the device); displacements within 1e-8 relative (FP64 path, both sides
solving tightly) and 1e-6 relative (mixed path).
"""
import numpy as np
import pytest

from _util import CFG, LPM, O, gpu_problem, hetero_plate, oracle_problem, oracle_step_args, rel

pytestmark = pytest.mark.gpu

K_TOL = 1e-12
FP64_DISP_TOL = 1e-8
MIXED_DISP_TOL = 1e-6


def small_cases():
    return {
        "hex": CFG.hex_plate(size=3.0, radius=0.1, steps=3, total_disp=0.003),
        "sc": CFG.sc_cube(size=2.4, radius=0.2, steps=3, total_disp=0.003),
        "sq": _square(),
        "fcc_j2": CFG.fcc_bar(size=(1.6, 1.6, 2.4), radius=0.2, steps=3, strain=0.02),
        "sc_j2": CFG.sc_cube(size=2.0, radius=0.25, steps=3, total_disp=0.06, ptype=LPM.ParticleType.J2Plasticity,
                             j2=(200.0, 0.0, 38714.0, 10.0)),
        # pre-cracked plate (explicit bond lists), loaded below the first bond break
        "hex_crack": CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=2, total_disp=0.001),
    }


def _square():
    c = CFG.hex_plate(size=2.0, radius=0.1, steps=2, total_disp=0.002)
    xyz = LPM.createPlateSQ2D(c.box, LPM.UnitCell(LPM.LatticeType.Square2D, 0.1))
    top = np.nonzero(xyz[:, 1] > c.box[3] - 0.2)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 1] < c.box[2] + 0.2)[0].astype(np.int32)
    c.lattice, c.xyz, c.types = LPM.LatticeType.Square2D, xyz, np.zeros(len(xyz), np.int32)
    c.groups = {"top": top, "bottom": bot}
    c.name = "sq2d"
    return c


CASES = small_cases()


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    return CASES[request.param]


def test_topology_bit_exact(case):
    g = gpu_problem(case)
    o = oracle_problem(case)
    t = g.topology()
    nb0, nb1, p2 = o.bonds()
    nconn, nlq, conns = o.conns()
    assert np.array_equal(t["nb0"], nb0)
    assert np.array_equal(t["nb1"], nb1)
    assert np.array_equal(t["bond_p2"], p2)
    assert np.array_equal(t["nconn"], nconn)
    assert np.array_equal(t["nlq"], nlq)
    assert np.array_equal(t["conns"], conns)
    Kp, IK, JK, K = g.export_csr()
    assert g.sizes["nnz_upper"] == o.export_csr()[0][-1]
    assert np.array_equal(Kp, o.export_csr()[0])


def test_initial_force_bit_exact(case):
    g = gpu_problem(case)
    o = oracle_problem(case)
    o.update_geometry()
    o.update_force_state()
    sg, so = g.state(), o.state()
    assert np.array_equal(sg["pin"], so["pin"])
    assert np.array_equal(sg["stress"], so["stress"])
    assert np.array_equal(sg["damage_visual"], so["damage_visual"])


@pytest.mark.parametrize("exact", [True, False], ids=["exact", "fast"])
def test_stiffness_matches(case, exact):
    """The bit-exact kernel reproduces the reference's K before the BC elimination bit for bit;
    the fast form (the default) agrees within K_TOL of max|K|, before and after the elimination."""
    g = gpu_problem(case)
    g.set_assembly_exact(exact)
    o = oracle_problem(case)
    o.update_geometry()
    o.update_force_state()
    disp, force = oracle_step_args(case, 0)
    o.apply_bc(disp, force)
    g.apply_load_step(case.load_step(0))
    for apply_bc in (False, True):
        o.assemble(apply_bc)
        g.assemble(apply_bc)
        Kp, IK, JK, K = g.export_csr()
        oKp, oIK, oJK, oK = o.export_csr()
        assert np.array_equal(IK, oIK)
        assert np.array_equal(JK, oJK)
        err = np.abs(K - oK).max() / np.abs(oK).max()
        assert err <= K_TOL, f"apply_bc={apply_bc}: max rel {err}"
        if not apply_bc and exact:
            assert np.array_equal(K, oK), "stiffness before the BC elimination should be bit-exact"


def test_linear_solve(case):
    g = gpu_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    o = oracle_problem(case, cg_rtol=1e-24, cg_atol=0.0)
    o.update_geometry()
    o.update_force_state()
    disp, force = oracle_step_args(case, 0)
    o.apply_bc(disp, force)
    g.apply_load_step(case.load_step(0))
    o.assemble(True)
    g.assemble(True)
    o.update_geometry()
    o.update_force_state()
    ro = o.update_rr()
    g.update_force_state()
    rg = g.update_rr()
    assert np.array_equal(g.residual(), o.residual())
    assert abs(rg - ro) <= 1e-14 * max(ro, 1e-300)
    xo, _ = o.cg()
    xg, st = g.solve_linear()
    assert rel(xg, xo) <= 1e-9, rel(xg, xo)
    assert st["cg_iters"] > 0


@pytest.mark.parametrize("precision,tol", [(0, FP64_DISP_TOL), (1, MIXED_DISP_TOL)])
def test_load_steps(case, precision, tol):
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(case, precision=precision, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    x0 = case.xyz
    for s in range(len(case.steps)):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg and oko
        sg, so = g.state(), o.state()
        e = rel(sg["xyz"] - x0, so["xyz"] - x0)
        assert e <= tol, f"step {s}: rel disp err {e}"
        assert abs(stg["reaction_norm"] - sto["reaction_norm"]) <= tol * sto["reaction_norm"] * 10
        if int(case.ptype) == 2:
            e_sv = rel(sg["state_var"], so["state_var"])
            assert e_sv <= 100 * tol, f"step {s}: state_var rel err {e_sv}"


def test_reference_tolerances_fp64():
    """The reference's own settings (CG 1e-12 on squared norms, Newton 1e-5): same Newton and
    close CG iteration counts, displacements close."""
    case = CFG.hex_plate(size=3.0, radius=0.1, steps=2, total_disp=0.002)
    g = gpu_problem(case)
    o = oracle_problem(case)
    o.update_geometry()
    o.update_force_state()
    for s in range(2):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg and oko
        assert stg["newton_solves"] == sto["newton_solves"]
        assert abs(stg["cg_iters"] - sto["cg_iters"]) <= 0.05 * sto["cg_iters"] + 3
        assert rel(g.state()["xyz"] - case.xyz, o.state()["xyz"] - case.xyz) <= 1e-5


def test_damage_bonds_break():
    """Brittle bonds (particle_elastic.h:52-68): the same bonds break in the same load steps."""
    case = CFG.hex_plate(size=2.0, radius=0.1, steps=3, total_disp=0.024, critical_bstrain=3e-3)
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(case, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    broke = 0
    for s in range(3):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg == oko
        bg, bo = g.state()["bdamage"], o.state()["bdamage"]
        assert np.array_equal(bg, bo), f"step {s}: broken bond sets differ"
        broke = int((bo == 1).sum())
        assert rel(g.state()["xyz"] - case.xyz, o.state()["xyz"] - case.xyz) <= FP64_DISP_TOL
    assert broke > 0, "the case should break some bonds"


def test_cut_back_matches():
    """A small Newton cap makes the full step fail; it is halved and retried
    (solver_static.h:78-87), with the same number of cuts as the oracle."""
    case = CFG.hex_plate(size=2.0, radius=0.1, steps=1, total_disp=0.01)
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9, max_iter=5)
    g = gpu_problem(case, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    okg, stg = g.solve_load_step(case.load_step(0))
    oko, sto = o.solve_load_step(*oracle_step_args(case, 0))
    assert okg == oko
    assert stg["cuts"] == sto["cuts"]
    if okg:
        assert rel(g.state()["xyz"] - case.xyz, o.state()["xyz"] - case.xyz) <= FP64_DISP_TOL


def test_precrack_grows_like_oracle():
    """The slit of a notched plate (bond exclusion, explicit bond lists) grows under tension:
    the same bonds break in the same load steps as in the oracle."""
    case = CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=8, total_disp=0.008)
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(case, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    for s in range(len(case.steps)):
        okg, stg = g.solve_load_step(case.load_step(s))
        oko, sto = o.solve_load_step(*oracle_step_args(case, s))
        assert okg == oko and stg["cuts"] == sto["cuts"]
        assert stg["newton_solves"] == sto["newton_solves"], f"step {s}"
        bg, bo = g.state()["bdamage"], o.state()["bdamage"]
        assert np.array_equal(bg == 1.0, bo == 1.0), f"step {s}: broken bond sets differ"
        assert rel(g.state()["xyz"] - case.xyz, o.state()["xyz"] - case.xyz) <= FP64_DISP_TOL
    assert (bo == 1.0).sum() > 100, "the crack should grow"


def _shuffled_bonds(case, seed):
    """The bond search's lists with each particle's layer-0 and layer-1 lists shuffled: bond
    files need not list partners in id order (Assembly::readBond keeps file order)."""
    nb0, nb1, p2 = CFG.bond_lists(case.xyz, LPM.UnitCell(case.lattice, case.radius))
    rng = np.random.default_rng(seed)
    p2 = p2.copy()
    start = 0
    for a, b in zip(nb0, nb1):
        p2[start:start + a] = rng.permutation(p2[start:start + a])
        p2[start + a:start + a + b] = rng.permutation(p2[start + a:start + a + b])
        start += a + b
    return nb0, nb1, p2


@pytest.mark.parametrize("lat", ["hex", "sc"])
def test_user_bond_order_is_kept(lat):
    """Explicit bond lists in arbitrary order: the device keeps the caller's order, so every
    bond-ordered sum (forces, stiffness) matches the oracle given the same lists bit for bit."""
    case = CASES[lat]
    case = CFG.Case(**{**case.__dict__, "bonds": _shuffled_bonds(case, 7)})
    g = gpu_problem(case)
    g.set_assembly_exact(True)
    o = oracle_problem(case)
    t = g.topology()
    nb0, nb1, p2 = case.bonds
    assert np.array_equal(t["bond_p2"], p2) and np.array_equal(t["nb0"], nb0)
    assert np.array_equal(t["conns"], o.conns()[2])
    o.update_geometry()
    o.update_force_state()
    assert np.array_equal(g.state()["pin"], o.state()["pin"])
    disp, force = oracle_step_args(case, 0)
    o.apply_bc(disp, force)
    g.apply_load_step(case.load_step(0))
    o.assemble(False)
    g.assemble(False)
    assert np.array_equal(g.export_csr()[3], o.export_csr()[3])


def test_bond_coefficients_and_initial_damage():
    """Per-bond Kn/Tv (a heterogeneous material) and initially broken bonds, passed through
    the optional per-bond arrays of the descriptor: forces bit-exact, load steps as the oracle."""
    case = hetero_plate()
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    g = gpu_problem(case, **kw)
    assert np.array_equal(g.state()["pin"], o.state()["pin"])
    assert np.array_equal(g.state()["damage_visual"], o.state()["damage_visual"])
    for s in range(len(case.steps)):
        okg, _ = g.solve_load_step(case.load_step(s))
        oko, _ = o.solve_load_step(*oracle_step_args(case, s))
        assert okg and oko
        assert rel(g.state()["xyz"] - case.xyz, o.state()["xyz"] - case.xyz) <= FP64_DISP_TOL
    assert np.array_equal(g.state()["bdamage"], o.state()["bdamage"])


def _asym_damage_plate():
    """A hexagonal plate whose explicit per-bond damage breaks 4% of the directed bonds in one
    direction only, so the opposite bonds stay intact (the case where the fast assembly takes
    the opposite bonds' own cosines)."""
    case = CFG.hex_plate(size=2.4, radius=0.1, steps=2, total_disp=0.002, tol_iter=1e-9)
    o = oracle_problem(case)
    nb0, nb1, p2 = o.bonds()
    kn, tv = o.bond_kntv()
    rng = np.random.default_rng(11)
    dmg = (rng.random(len(p2)) < 0.04).astype(np.float64)
    dmg[rng.random(len(p2)) < 0.05] = 0.5  # partial damage too
    case.bonds = (nb0, nb1, p2)
    case.bond_props = (kn, tv, dmg)
    case.name = "hex_asym_damage"
    return case


@pytest.mark.parametrize("name", ["hex", "sc", "sq", "fcc_j2", "sc_j2", "hex_crack", "asym"])
def test_fast_assembly_matches_exact_after_loading(name):
    """The fast stiffness form against the bit-exact kernel on deformed, yielded and damaged
    states: after two load steps each handle re-assembles from the same state, before and after
    the BC elimination, within K_TOL of max|K|; the oracle's K of the same state agrees too."""
    case = _asym_damage_plate() if name == "asym" else CASES[name]
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(case, **kw)
    o = oracle_problem(case, **kw)
    o.update_geometry()
    o.update_force_state()
    for s in range(min(2, len(case.steps))):
        assert g.solve_load_step(case.load_step(s))[0]
        assert o.solve_load_step(*oracle_step_args(case, s))[0]
    for apply_bc in (False, True):
        g.set_assembly_exact(True)
        g.assemble(apply_bc)
        Ke = g.export_csr()[3]
        g.set_assembly_exact(False)
        g.assemble(apply_bc)
        Kf = g.export_csr()[3]
        o.assemble(apply_bc)
        oK = o.export_csr()[3]
        scale = np.abs(Ke).max()
        assert np.abs(Kf - Ke).max() <= K_TOL * scale, (apply_bc, np.abs(Kf - Ke).max() / scale)
        assert np.abs(Kf - oK).max() <= 1e-9 * scale  # the states differ by the solves' rounding


TANGENT_CASES = {
    "fcc_j2": lambda: CFG.fcc_bar(size=(1.6, 1.6, 2.4), radius=0.2, steps=3, strain=0.02),
    "hex_crack": lambda: CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=6, total_disp=0.006),
}


@pytest.mark.parametrize("name", sorted(TANGENT_CASES))
@pytest.mark.parametrize("precision,tol", [(0, FP64_DISP_TOL), (1, MIXED_DISP_TOL)])
def test_tangent_mode_matches_oracle(name, precision, tol):
    """Tangent mode (K re-assembled from the current state before every Newton solve): the
    device against the oracle in the same mode, itself pinned to the reference's own Newton
    loop and stiffness calls (golden fixtures fcc_j2_tangent, hex_crack_tangent)."""
    case = TANGENT_CASES[name]()
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9, tangent=True)
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
            assert np.array_equal(g.state()["bdamage"] == 1.0, o.state()["bdamage"] == 1.0)
        e = rel(g.state()["xyz"] - case.xyz, o.state()["xyz"] - case.xyz)
        assert e <= tol, f"step {s}: rel disp err {e}"
    if precision == 0:
        K, oK = g.export_csr()[3], o.export_csr()[3]
        assert np.abs(K - oK).max() <= 1e-12 * np.abs(oK).max()


def test_bond_list_overflow_is_a_topology_error():
    """More bonds on one particle than the fixed per-particle staging holds (32) is rejected
    with LPMGPU_ERR_TOPOLOGY, not truncated."""
    c = CFG.hex_plate(size=2.0, radius=0.1, steps=1, total_disp=0.001)
    nb0, nb1, p2 = CFG.bond_lists(c.xyz, LPM.UnitCell(c.lattice, c.radius))
    nb0, nb1 = nb0.copy(), nb1.copy()
    extra = np.arange(1, 34, dtype=np.int32)  # particle 0 claims 33 layer-1 partners
    start1 = int(nb0[0])
    p2 = np.concatenate([p2[:start1], extra, p2[int(nb0[0] + nb1[0]):]]).astype(np.int32)
    nb1[0] = len(extra)
    ass = c.assembly()
    ass.bonds = (nb0, nb1, p2)
    with pytest.raises(LPM.LpmGpuError) as e:
        LPM.GpuProblem(ass)
    assert e.value.status == 7


def test_step_without_boundary_conditions_is_a_no_op():
    """A load step with no displacement or force condition leaves a body at rest: Newton
    converges before any linear solve, on the device and in the oracle."""
    c = CFG.hex_plate(size=2.0, radius=0.1, steps=1, total_disp=0.001)
    g = gpu_problem(c)
    o = oracle_problem(c)
    o.update_geometry()
    o.update_force_state()
    okg, stg = g.solve_load_step(LPM.LoadStep())
    oko, sto = o.solve_load_step([], [])
    assert okg and oko
    assert stg["newton_solves"] == sto["newton_solves"] == 0
    assert np.array_equal(g.state()["xyz"], c.xyz)


@pytest.mark.parametrize("size", [0.4, 0.6])
def test_tiny_plates_match_oracle(size):
    """Plates of 4 and 12 particles (rows shorter than a slice, every particle on the boundary)."""
    c = CFG.hex_plate(size=size, radius=0.1, steps=2, total_disp=0.002)
    kw = dict(cg_rtol=1e-24, cg_atol=0.0, tol_iter=1e-9)
    g = gpu_problem(c, **kw)
    o = oracle_problem(c, **kw)
    o.update_geometry()
    o.update_force_state()
    t = g.topology()
    assert np.array_equal(t["conns"], o.conns()[2])
    for s in range(2):
        okg, _ = g.solve_load_step(c.load_step(s))
        oko, _ = o.solve_load_step(*oracle_step_args(c, s))
        assert okg == oko
        if okg:
            assert rel(g.state()["xyz"] - c.xyz, o.state()["xyz"] - c.xyz) <= FP64_DISP_TOL
