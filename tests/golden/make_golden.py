"""Generates the golden fixtures in this directory from the reference's own hot path.

    python tests/golden/make_golden.py        (needs oracle/_ref/lpm_ref: make -C oracle ref)

Each case is a small problem from lpm-cpp_b200/configs.py.  The reference (LPM-CPP headers
compiled unmodified against the oracle/shim MKL stand-in, run single-threaded so every sum has
one order) generates the lattice itself, builds bonds and connections, assembles, and runs
SolverStatic::solveProblem's step loop (fatigue cases: SolverFatigue::solveProblemStatic for the
load steps, then the cycles of solveProblemCyclic); its outputs are stored as compressed .npz:
  xyz0, nb0, nb1, bond_p2, nconn, nlq, conns          topology
  K_pointer, IK, JK, K                                the reference CSR after load step 0 (dump_k)
  xyz_<s>, pin_<s>, state_var_<s>, bdamage_<s>        state after each load step (or cycle)
  steps                                               [newton_solves, cg_iters, cuts, reaction_norm]
  cycles                                              fatigue: [N, dNdt] after each cycle
"""
from __future__ import annotations

import importlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

sys.path.insert(0, os.path.dirname(HERE))
from _util import hetero_plate  # noqa: E402

CFG = importlib.import_module("lpm-cpp_b200.configs")
LPM = importlib.import_module("lpm-cpp_b200.lpm")


def square_plate():
    c = CFG.hex_plate(size=1.6, radius=0.1, steps=2, total_disp=0.002)
    xyz = LPM.createPlateSQ2D(c.box, LPM.UnitCell(LPM.LatticeType.Square2D, 0.1))
    top = np.nonzero(xyz[:, 1] > c.box[3] - 0.2)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 1] < c.box[2] + 0.2)[0].astype(np.int32)
    c.lattice, c.xyz, c.types = LPM.LatticeType.Square2D, xyz, np.zeros(len(xyz), np.int32)
    c.groups = {"top": top, "bottom": bot}
    return c


def bcc_block():
    c = CFG.sc_cube(size=1.6, radius=0.2, steps=2, total_disp=0.002)
    cell = LPM.UnitCell(LPM.LatticeType.BCC3D, 0.2)
    xyz = LPM.createCuboidBCC3D(c.box, cell)
    top = np.nonzero(xyz[:, 2] > c.box[5] - 0.4)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 2] < c.box[4] + 0.4)[0].astype(np.int32)
    zb = xyz[bot]
    c0 = bot[np.lexsort((zb[:, 2], zb[:, 1], zb[:, 0]))[0]]
    c1 = bot[np.lexsort((zb[:, 2], zb[:, 1], -zb[:, 0]))[0]]
    c.lattice, c.xyz, c.types = LPM.LatticeType.BCC3D, xyz, np.zeros(len(xyz), np.int32)
    c.groups = {"top": top, "bottom": bot, "corner0": np.array([c0], np.int32), "corner1": np.array([c1], np.int32)}
    return c


def cases():
    """name -> (case builder, reference options).  The builders are what the tests call too."""
    return {
        "hex_small": (lambda: CFG.hex_plate(size=3.0, radius=0.1, steps=3, total_disp=0.003), {"dump_k": (0,)}),
        "sc_small": (lambda: CFG.sc_cube(size=1.6, radius=0.2, steps=2, total_disp=0.002), {"dump_k": (0,)}),
        "sq_small": (square_plate, {"dump_k": (0,)}),
        "bcc_small": (bcc_block, {"dump_k": (0,)}),
        "fcc_j2": (lambda: CFG.fcc_bar(size=(1.2, 1.2, 1.6), radius=0.2, steps=3, strain=0.02), {}),
        "sc_j2": (lambda: CFG.sc_cube(size=2.0, radius=0.25, steps=3, total_disp=0.06,
                                      ptype=LPM.ParticleType.J2Plasticity, j2=(200.0, 0.0, 38714.0, 10.0)), {}),
        "hex_damage": (lambda: CFG.hex_plate(size=2.0, radius=0.1, steps=3, total_disp=0.024, critical_bstrain=3e-3,
                                             tol_iter=1e-9), {"cg_tol": (1e-24, 0.0)}),
        # pre-crack by bond exclusion, built by the reference through readDump + readBond
        "hex_crack": (lambda: CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=8, total_disp=0.008,
                                                tol_iter=1e-9), {"cg_tol": (1e-24, 0.0), "dump_k": (0,)}),
        # per-bond Kn/Tv and initially broken bonds written into the bonds (bond.h:25-27)
        "hex_hetero": (hetero_plate, {"cg_tol": (1e-24, 0.0), "dump_k": (0,)}),
        # tangent mode: the stiffness re-assembled before every Newton solve (driver directive
        # "tangent 1", the reference's own Newton loop and stiffness calls re-ordered)
        "fcc_j2_tangent": (lambda: CFG.fcc_bar(size=(1.2, 1.2, 1.6), radius=0.2, steps=3, strain=0.02),
                           {"cg_tol": (1e-24, 0.0), "tangent": True, "dump_k": (2,)}),
        "hex_crack_tangent": (lambda: CFG.notched_plate(size=2.0, radius=0.1, crack=0.3, steps=6, total_disp=0.006,
                                                        tol_iter=1e-9), {"cg_tol": (1e-24, 0.0), "tangent": True}),
        # ParticleElasticDamage with the nonlocal damage rate (searchNonlocalNeighbors + the
        # averaging of SolverStatic::updateStaticDamage): damage grows in every step
        "hex_edamage": (lambda: CFG.edamage_plate(), {"cg_tol": (1e-24, 0.0), "dump_k": (1,)}),
        # undamaged grips (type 3): no damage there, and left out of the nonlocal averaging
        "hex_edamage_grips": (lambda: CFG.edamage_plate(undamaged_band=0.5), {"cg_tol": (1e-24, 0.0), "dump_k": (1,)}),
        # FCC with cubic elastic constants (setParticleProperty's (C11, C12, C44) overload, as ex3)
        "fcc_cubic": (lambda: CFG.fcc_cubic_cube(), {"cg_tol": (1e-24, 0.0), "dump_k": (0,)}),
        # SolverFatigue: one static step, then four cycles (two steps up, two down) of HCF damage
        "hex_fatigue": (lambda: CFG.fatigue_plate(), {"cg_tol": (1e-24, 0.0), "fatigue": True}),
        # the exponential time map: dN/dt = (int)(1/tau exp(t/tau)) is 0, 0, 1, 2, 3 at tau = 2
        "hex_fatigue_exp": (lambda: CFG.fatigue_plate(cycles=4, tmode="exponential", tau=2.0, A=40.0),
                            {"cg_tol": (1e-24, 0.0), "fatigue": True}),
        # undamaged grips (type 3 near the top and bottom edges), as ex5_isoelasticity_2d_fatigue
        "hex_fatigue_grips": (lambda: CFG.fatigue_plate(undamaged_band=0.5), {"cg_tol": (1e-24, 0.0), "fatigue": True}),
        # the LoadCTForce cycle: middle row held in y, top and bottom edges pulled apart
        "hex_fatigue_ct": (lambda: CFG.fatigue_plate(load_type="ct_force", amplitude=250.0, cycles=4, tol_iter=1e-7),
                           {"cg_tol": (1e-24, 0.0), "fatigue": True}),
        # 3D: a simple-cubic cube under the LoadDogBoneDisp cycle (as ex5_isoelasticity_3d_fatigue)
        "sc_fatigue_dogbone": (lambda: CFG.fatigue_cube(), {"cg_tol": (1e-24, 0.0), "fatigue": True}),
        # the LoadUniaxialForce cycle: the top edge pulled by a shared force (force BCs in fatigue)
        "hex_fatigue_force": (lambda: CFG.fatigue_plate(load_type="uniaxial_force", amplitude=200.0, cycles=4,
                                                        tol_iter=1e-7),
                              {"cg_tol": (1e-24, 0.0), "fatigue": True}),
    }


def make(name, build, opts):
    case = build()
    d = tempfile.mkdtemp(prefix=f"golden_{name}_")
    try:
        tangent = bool(opts.get("tangent", False))
        spec = O.write_ref_spec(case, d, cg_tol=opts.get("cg_tol"), dump_k=opts.get("dump_k", ()),
                                loop="step" if tangent else "ref", tangent=tangent)
        O.run_ref(spec, d, threads=1)
        rb = lambda f, t: O.read_bin(d, f, t)  # noqa: E731
        out = {"xyz0": rb("xyz0.f64", np.float64).reshape(-1, 3)}
        for f in ("nb0", "nb1", "bond_p2", "nconn", "nlq", "conns"):
            out[f] = rb(f + ".i32", np.int32)
        for s in opts.get("dump_k", ()):
            tag = "%03d" % s
            out["K_pointer"] = rb(f"K_pointer_{tag}.i64", np.int64)
            out["IK"] = rb(f"IK_{tag}.i64", np.int64)
            out["JK"] = rb(f"JK_{tag}.i64", np.int64)
            out["K"] = rb(f"K_{tag}.f64", np.float64)
        rows = O.read_ref_steps(d)
        out["steps"] = np.array([[r["newton_solves"], r["cg_iters"], r["cuts"], r["reaction_norm"]] for r in rows])
        for s in range(len(rows)):
            tag = "%03d" % s
            out[f"xyz_{s}"] = rb(f"xyz_{tag}.f64", np.float64).reshape(-1, 3)
            out[f"pin_{s}"] = rb(f"pin_{tag}.f64", np.float64).reshape(-1, 3)
            if int(case.ptype) == 2:
                out[f"state_var_{s}"] = rb(f"state_var_{tag}.f64", np.float64).reshape(-1, 7)
            if int(case.ptype) == 3:
                out[f"state_var_{s}"] = rb(f"state_var_{tag}.f64", np.float64).reshape(-1, 3)
                out[f"damage_{s}"] = rb(f"damage_{tag}.f64", np.float64)
                out[f"bdamage_{s}"] = rb(f"bdamage_{tag}.f64", np.float64)
            if int(case.ptype) == 1:
                out[f"state_var_{s}"] = rb(f"state_var_{tag}.f64", np.float64).reshape(-1, 1)
                out[f"damage_{s}"] = rb(f"damage_{tag}.f64", np.float64)
                out[f"bdamage_{s}"] = rb(f"bdamage_{tag}.f64", np.float64)
            if case.material.critical_bstrain < 1.0 or case.bond_props is not None:
                out[f"bdamage_{s}"] = rb(f"bdamage_{tag}.f64", np.float64)
        if opts.get("fatigue"):
            # cycle count N and dNdt after each cycle of SolverFatigue::solveProblemCyclic
            out["cycles"] = np.loadtxt(os.path.join(d, "cycles.txt"), ndmin=2)
        out["meta"] = np.array(json.dumps({"name": name,
                                           "opts": {k: (list(v) if isinstance(v, tuple) else v) for k, v in opts.items()},
                                           "n": int(case.n), "spec": spec}))
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **out)
        return path, os.path.getsize(path)
    finally:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    if not O.ref_available():
        sys.exit("oracle/_ref/lpm_ref is not built (make -C oracle ref)")
    only = set(sys.argv[1:])
    for name, (build, opts) in cases().items():
        if only and name not in only:
            continue
        p, sz = make(name, build, opts)
        print(f"{name}: {sz / 1024:.0f} KiB -> {os.path.relpath(p, ROOT)}")
