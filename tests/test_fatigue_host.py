"""Host side of SolverFatigue (no device): the Python mirror's load cycles and time maps against
the reference's definitions, its readLoad, and the C ABI's argument checks of the fatigue entry
points.  The device steps are checked against the oracle in test_solver_fatigue.py."""
import ctypes as C
import math

import numpy as np

from _util import CFG, LPM, fatigue_cycles


def _bcs(step):
    return ([(tuple(b.group), b.flag, b.step) for b in step.dispBCs],
            [(tuple(b.group), b.fx, b.fy, b.fz) for b in step.forceBCs])


def test_load_cycle_types_follow_load_step_fatigue():
    """generateLoadCycle (solver_fatigue.h:128-180) with the four load-step templates of
    include/load_step_fatigue.h: n_interval steps up by (f1 - f0) / n, then n down by (f2 - f1) / n."""
    g0, g1, g2 = (np.array([k, k + 10], np.int32) for k in range(3))
    spec = [0.5, 2.5, 1.0, 3.0, 0.0]
    T = LPM.FatigueLoadType
    for N, (f0, f1, f2) in ((0, (0.5, 2.5, 1.0)), (1, (1.0, 3.0, 0.0))):
        up, down = (f1 - f0) / 4, (f2 - f1) / 4
        for v, step in zip([up] * 4 + [down] * 4, LPM.generateLoadCycle(T.LoadUniaxialDisp, spec, N, 4, [g0, g1, g2])):
            assert _bcs(step) == ([(tuple(g0), "x", 0.0), (tuple(g1), "y", v), (tuple(g2), "y", 0.0)], [])
        for v, step in zip([up] * 4 + [down] * 4, LPM.generateLoadCycle(T.LoadUniaxialForce, spec, N, 4, [g0, g1, g2])):
            assert _bcs(step) == ([(tuple(g0), "x", 0.0), (tuple(g2), "y", 0.0)], [(tuple(g1), 0.0, v, 0.0)])
        for v, step in zip([up] * 4 + [down] * 4, LPM.generateLoadCycle(T.LoadDogBoneDisp, spec, N, 4, [g0, g1])):
            assert _bcs(step) == ([(tuple(g0), "x", 0), (tuple(g0), "y", v), (tuple(g0), "z", 0),
                                   (tuple(g1), "x", 0.0), (tuple(g1), "y", 0.0), (tuple(g1), "z", 0.0)], [])
        for v, step in zip([up] * 4 + [down] * 4, LPM.generateLoadCycle(T.LoadCTForce, spec, N, 4, [g0, g1, g2])):
            assert _bcs(step) == ([(tuple(g0), "y", 0.0), (tuple(g1), "x", 0.0), (tuple(g2), "x", 0.0)],
                                  [(tuple(g1), 0.0, v, 0.0), (tuple(g2), 0.0, -v, 0.0)])


def test_time_maps_truncate_like_the_reference():
    """func_dNdt_linear / func_dNdt_exponental (solver_fatigue.h:60-68) cast to int."""
    assert LPM.func_dNdt_linear(1e-4) == int(1 / 1e-4)
    assert LPM.func_dNdt_linear(0.3) == 3
    assert [LPM.func_dNdt_exponental(2.0, t) for t in range(5)] == [0, 0, 1, 2, 3]
    assert LPM.func_dNdt_exponental(0.5, 1.0) == int(2 * math.exp(2.0))


def test_cycle_count_follows_the_spectrum():
    """solveProblemCyclic's loop runs while N < (len(spectrum) - 1) / 2, with N += dN/dt."""
    c = CFG.fatigue_plate(cycles=8, tau=0.5)
    assert [N for N, _, _ in fatigue_cycles(c)] == [2, 4, 6, 8]
    c = CFG.fatigue_plate(cycles=4, tmode="exponential", tau=2.0)
    assert [(N, d) for N, d, _ in fatigue_cycles(c)] == [(0, 0), (0, 0), (1, 1), (3, 2), (6, 3)]


def test_read_load_appends_every_number(tmp_path):
    p = tmp_path / "load.txt"
    p.write_text("0\n1.5 0\n  2.5e-1\n0\n")
    s = LPM.SolverFatigue.__new__(LPM.SolverFatigue)
    s.load_spectrum = []
    LPM.SolverFatigue.readLoad(s, str(p))
    assert s.load_spectrum == [0.0, 1.5, 0.0, 0.25, 0.0]


def test_fatigue_entry_points_reject_bad_arguments():
    L = LPM.lib()
    st = LPM.Stats()
    flag = C.c_int32()
    assert L.lpmgpu_fatigue_solve_step(None, None, C.byref(st)) == 1
    assert L.lpmgpu_fatigue_static_step(None, None, C.byref(st)) == 1
    assert L.lpmgpu_fatigue_update_damage(None, 1.0, C.byref(flag)) == 1
    assert L.lpmgpu_fatigue_cycle(None, None, 0, 1.0, C.byref(st), C.byref(flag)) == 1


def test_fatigue_desc_fields_reach_the_c_struct():
    """The mirror packs the HCF rate law into lpmgpu_desc (appended after the elastic-damage
    fields, so earlier fields keep their offsets)."""
    c = CFG.fatigue_plate(A=7.0, B=2.5, d=0.75)
    d, _ = LPM._pack_desc(c.assembly())
    assert d.ptype == int(LPM.ParticleType.FatigueHCF) == 3
    assert (d.fatigue_A, d.fatigue_B, d.fatigue_d) == (7.0, 2.5, 0.75)
    assert LPM.Desc.fatigue_A.offset > LPM.Desc.damage_threshold.offset


def test_set_particle_property_per_type():
    """Assembly.setParticleProperty takes each particle type's isotropic argument list."""
    c = CFG.fatigue_plate()
    a = c.assembly()
    a.setParticleProperty(6.0, True, 71.7e3, 0.306, 2.003e-5, 2.833, 0.5, 1.0, 1.108)
    m = a.material
    assert (m.nonlocal_L, m.plane_stress, m.E, m.mu) == (6.0, True, 71.7e3, 0.306)
    assert (m.fatigue_A, m.fatigue_B, m.fatigue_d, m.damage_threshold, m.fatigue_limit_ratio) == \
        (2.003e-5, 2.833, 0.5, 1.0, 1.108)
    e = CFG.edamage_plate().assembly()
    e.setParticleProperty(0.3, True, 69e3, 0.3, 0.02, 0.5, 10.0, 0.9)
    assert (e.material.k0, e.material.k1, e.material.comp_tensile_ratio, e.material.damage_threshold) == \
        (0.02, 0.5, 10.0, 0.9)


def test_solver_modes_map_to_cg_tolerances():
    """SolverMode.CG keeps the reference CG's test; PARDISO (a direct solve) runs the device CG
    to 1e-12 relative; explicit tolerances win."""
    assert LPM._cg_tolerances(LPM.SolverMode.CG, None, None) == (1e-12, 1e-12)
    assert LPM._cg_tolerances(LPM.SolverMode.PARDISO, None, None) == (1e-24, 0.0)
    assert LPM._cg_tolerances(LPM.SolverMode.PARDISO, 1e-20, 1e-30) == (1e-20, 1e-30)


def test_set_particle_property_cubic_overload():
    """The (C11, C12, C44) overloads (particle_elastic.h:111, particle_elastic_damage.h:219) are
    taken when the second argument is a number, and reach lpmgpu_desc."""
    c = CFG.fcc_cubic_cube()
    a = c.assembly()
    a.setParticleProperty(0.5, 108e3, 61e3, 29e3, 0.01)
    m = a.material
    assert (m.C11, m.C12, m.C44, m.critical_bstrain, m.nonlocal_L) == (108e3, 61e3, 29e3, 0.01, 0.5)
    d, _ = LPM._pack_desc(a)
    assert (d.C11, d.C12, d.C44) == (108e3, 61e3, 29e3)
    e = CFG.edamage_plate().assembly()
    e.setParticleProperty(0.3, 90e3, 40e3, 25e3, 0.02, 0.5, 10.0, 0.9)
    assert (e.material.C11, e.material.k0, e.material.damage_threshold) == (90e3, 0.02, 0.9)
    a.setParticleProperty(0.5, False, 69e3, 0.3, 1.0)  # a bool: the isotropic overload
    assert a.material.C11 == 0.0 and a.material.E == 69e3
