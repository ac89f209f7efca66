"""Shared helpers: build the same problem in the CPU oracle and on the device."""
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

LPM = importlib.import_module("lpm-cpp_b200.lpm")
CFG = importlib.import_module("lpm-cpp_b200.configs")

LAT_NAME = {0: "sq2d", 1: "hex2d", 2: "sc3d", 3: "fcc3d", 4: "bcc3d"}


def oracle_problem(case, cg_rtol=1e-12, cg_atol=1e-12, tol_iter=None, max_iter=None, tangent=False):
    m = case.material
    mat = O.Material(ptype={2: "j2", 1: "elastic_damage", 3: "fatigue_hcf"}.get(int(case.ptype), "elastic"),
                     plane_stress=m.plane_stress, E=m.E, mu=m.mu,
                     critical_bstrain=m.critical_bstrain, sigmay=m.sigmay, xi=m.xi, H=m.H, A=m.A,
                     nonlocal_L=m.nonlocal_L, k0=m.k0, k1=m.k1, comp_tensile_ratio=m.comp_tensile_ratio,
                     damage_threshold=m.damage_threshold, fatigue_A=m.fatigue_A, fatigue_B=m.fatigue_B,
                     fatigue_d=m.fatigue_d, fatigue_limit_ratio=m.fatigue_limit_ratio, C11=m.C11, C12=m.C12,
                     C44=m.C44)
    o = O.OracleProblem(LAT_NAME[int(case.lattice)], case.radius, case.xyz, mat, types=case.types,
                        undamaged_type=case.undamaged_type,
                        max_iter=case.max_iter if max_iter is None else max_iter,
                        tol_iter=case.tol_iter if tol_iter is None else tol_iter, cg_rtol=cg_rtol, cg_atol=cg_atol,
                        bonds=getattr(case, "bonds", None), tangent=tangent,
                        nonlocal_cutoff_ratio=getattr(case, "nonlocal_cutoff_ratio", 0.0))
    if getattr(case, "bond_props", None) is not None:
        kn, tv, dmg = case.bond_props
        o.set_bond_kntv(kn, tv)
        o.set_bond_damage(dmg)
    return o


def hetero_plate(size=2.4, steps=3, total_disp=0.003, seed=3):
    """Hexagonal plate whose bonds carry their own Kn/Tv, drawn in [0.6, 1.4] x the values
    setParticleProperty gives (one factor per particle pair), with 3% of the pairs broken before
    loading: the per-bond properties an LPM-CPP example writes into its bonds (bond.h:25-27)."""
    case = CFG.hex_plate(size=size, radius=0.1, steps=steps, total_disp=total_disp, tol_iter=1e-9)
    o = oracle_problem(case)
    nb0, nb1, p2 = o.bonds()
    owner = np.repeat(np.arange(case.n), nb0 + nb1)
    key = np.minimum(owner, p2).astype(np.int64) * case.n + np.maximum(owner, p2)
    uniq, inv = np.unique(key, return_inverse=True)
    rng = np.random.default_rng(seed)
    factor = rng.uniform(0.6, 1.4, len(uniq))[inv]
    broken = (rng.random(len(uniq)) < 0.03)[inv].astype(np.float64)
    kn, tv = o.bond_kntv()
    case.bonds = (nb0, nb1, p2)  # per-bond arrays are sized and ordered by explicit lists
    case.bond_props = (kn * factor, tv * factor, broken)
    case.name = "hex_hetero"
    return case


def gpu_problem(case, precision=0, cg_rtol=1e-12, cg_atol=1e-12, tol_iter=None, max_iter=None, tangent=False):
    return LPM.GpuProblem(case.assembly(), undamaged_pt_type=case.undamaged_type, tangent=tangent,
                          max_iter=case.max_iter if max_iter is None else max_iter,
                          tol_iter=case.tol_iter if tol_iter is None else tol_iter,
                          precision=LPM.Precision(precision), cg_rtol=cg_rtol, cg_atol=cg_atol)


def oracle_step_args(case, s):
    disp, force = case.steps[s]
    flag = {"x": 0, "y": 1, "z": 2}
    return ([(case.groups[g], flag[f], v) for g, f, v in disp],
            [(case.groups[g], fx, fy, fz) for g, fx, fy, fz in force])


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def oracle_load_args(step):
    """A product-side LoadStep as the oracle's (disp, force) tuples."""
    flag = {"x": 0, "y": 1, "z": 2}
    return ([(np.asarray(b.group, np.int32), flag[b.flag], b.step) for b in step.dispBCs],
            [(np.asarray(b.group, np.int32), b.fx, b.fy, b.fz) for b in step.forceBCs])


def fatigue_disp_scale(case):
    """A displacement scale for comparing fatigue states: the spectrum's amplitude for a
    displacement-driven cycle, the particle radius for a force-driven one."""
    fat = case.meta["fatigue"]
    if fat["load_type"].endswith("disp"):
        return max(abs(v) for v in fat["spectrum"])
    return case.radius


def fatigue_cycles(case):
    """The cycles of SolverFatigue::solveProblemCyclic (solver_fatigue.h:183-218) for a fatigue
    case: yields (cycle count N after the cycle, dNdt, the cycle's LoadSteps)."""
    fat = case.meta["fatigue"]
    spec = fat["spectrum"]
    groups = [case.groups[g] for g in fat["groups"]]
    ltype = {"uniaxial_disp": LPM.FatigueLoadType.LoadUniaxialDisp,
             "uniaxial_force": LPM.FatigueLoadType.LoadUniaxialForce,
             "dogbone_disp": LPM.FatigueLoadType.LoadDogBoneDisp,
             "ct_force": LPM.FatigueLoadType.LoadCTForce}[fat["load_type"]]
    n_cycles = 0.5 * (len(spec) - 1)
    t, N = 0.0, 0
    while True:
        steps = LPM.generateLoadCycle(ltype, spec, N, fat["n_interval"], groups)
        if fat["tmode"] == "linear":
            dNdt = LPM.func_dNdt_linear(fat["tau"])
        else:
            dNdt = LPM.func_dNdt_exponental(fat["tau"], t)
            t += 1
        N += int(dNdt)
        yield N, dNdt, steps
        if not N < n_cycles:
            break
