"""Synthetic LPM workloads: lattices from the reference's generators, the boundary groups and
load paths of the reference examples, sized as the benchmark configurations.

A ``Case`` is plain data (coordinates, particle types, material, groups, load steps) so the
same problem can be handed to the device solver and to the CPU oracle.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional, Tuple

import numpy as np

from . import lpm as L

# (group name, flag 'x'|'y'|'z', step)  /  (group name, fx, fy, fz)
DispSpec = Tuple[str, str, float]
ForceSpec = Tuple[str, float, float, float]


@dataclass
class Case:
    name: str
    lattice: L.LatticeType
    radius: float
    box: List[float]
    xyz: np.ndarray
    ptype: L.ParticleType
    material: L.Material
    types: np.ndarray
    groups: Dict[str, np.ndarray]
    steps: List[Tuple[List[DispSpec], List[ForceSpec]]]
    undamaged_type: int = -1
    max_iter: int = 30
    tol_iter: float = 1e-5
    euler: Tuple[int, Tuple[float, float, float]] = (0, (0.0, 0.0, 0.0))
    meta: dict = field(default_factory=dict)
    # explicit bond lists (nb0, nb1, p2) as Assembly::readBond builds them; None -> bond search
    bonds: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None
    # per-bond (Kn, Tv, bdamage) in bond order, written into the bonds before the first force
    # update (a heterogeneous material, initial damage); None -> setParticleProperty's values
    bond_props: Optional[Tuple[np.ndarray, np.ndarray, np.ndarray]] = None
    # > 0: Assembly::searchNonlocalNeighbors(cutoff_ratio) before solving (nonlocal damage)
    nonlocal_cutoff_ratio: float = 0.0

    @property
    def n(self):
        return len(self.xyz)

    @property
    def dim(self):
        return 2 if self.lattice in (L.LatticeType.Square2D, L.LatticeType.Hexagon2D) else 3

    def load_step(self, s: int) -> L.LoadStep:
        disp, force = self.steps[s]
        st = L.LoadStep()
        for g, flag, step in disp:
            st.dispBCs.append(L.DispBC(self.groups[g], L.LoadMode.Relative, flag, step))
        for g, fx, fy, fz in force:
            st.forceBCs.append(L.ForceBC(self.groups[g], L.LoadMode.Relative, fx, fy, fz))
        return st

    def assembly(self) -> L.Assembly:
        a = L.Assembly(self.xyz, self.box, L.UnitCell(self.lattice, self.radius), self.ptype)
        a.type = self.types.copy()
        a.material = self.material
        a.bonds = self.bonds
        if self.bond_props is not None:
            a.bond_kn, a.bond_tv, a.bond_damage = self.bond_props
        if self.nonlocal_cutoff_ratio > 0:
            a.searchNonlocalNeighbors(self.nonlocal_cutoff_ratio)
        return a


def bond_lists(xyz: np.ndarray, cell: L.UnitCell,
               exclude: Optional[Callable[[np.ndarray, np.ndarray], np.ndarray]] = None):
    """Bond lists of Assembly::createBonds (include/assembly.h:213-234) built on the host, for
    problems whose bonds are prepared before the solver sees them: a bond i-j for every pair with
    distance < 1.01*cutoff[1], layer 0 below 1.01*cutoff[0]; per particle the layer-0 partners,
    then the layer-1 partners, each in ascending id.  ``exclude(i, j)`` (arrays, i < j) marks
    bonds to leave out, as the reference's geometry tools do for notches and cracks
    (geometry/geo1_CT_configuration.cpp:79-134); the decision is taken once per pair, so the
    lists stay symmetric.  Returns (nb0, nb1, p2) in int32."""
    from scipy.spatial import cKDTree

    xyz = np.ascontiguousarray(xyz, dtype=np.float64)
    n = len(xyz)
    rc0, rc1 = 1.01 * cell.neighbor_cutoff[0], 1.01 * cell.neighbor_cutoff[1]
    pairs = cKDTree(xyz).query_pairs(rc1, output_type="ndarray").astype(np.int64)
    i, j = pairs[:, 0], pairs[:, 1]
    dv = xyz[i] - xyz[j]
    d = np.sqrt(dv[:, 0] * dv[:, 0] + dv[:, 1] * dv[:, 1] + dv[:, 2] * dv[:, 2])
    keep = d < rc1
    if exclude is not None:
        keep &= ~np.asarray(exclude(i, j), dtype=bool)
    i, j, d = i[keep], j[keep], d[keep]
    layer = np.where(d < rc0, 0, 1)
    p1, p2, ly = np.concatenate([i, j]), np.concatenate([j, i]), np.concatenate([layer, layer])
    order = np.lexsort((p2, ly, p1))
    nb0 = np.bincount(p1[ly == 0], minlength=n).astype(np.int32)
    nb1 = np.bincount(p1[ly == 1], minlength=n).astype(np.int32)
    return nb0, nb1, p2[order].astype(np.int32)


def slit_exclusion(xyz: np.ndarray, y_slit: float, x_from: float, x_to: float):
    """exclude(i, j) for a zero-width straight slit on y = y_slit between x_from and x_to: a
    bond is cut when its segment crosses the slit line inside that span."""
    xyz = np.asarray(xyz)

    def exclude(i, j):
        yi, yj = xyz[i, 1] - y_slit, xyz[j, 1] - y_slit
        cross = yi * yj < 0
        t = np.where(cross, yi / np.where(cross, yi - yj, 1.0), 0.0)
        xc = xyz[i, 0] + t * (xyz[j, 0] - xyz[i, 0])
        return cross & (xc >= x_from) & (xc <= x_to)

    return exclude


def _gen(lattice, radius, box, euler=(0, (0.0, 0.0, 0.0))):
    cell = L.UnitCell(lattice, radius)
    R = L.createRMatrix(euler[0], euler[1])
    return L._generate(lattice, box, cell, R)


def hex_plate(size=10.0, radius=0.1, E=69e3, mu=0.3, plane_stress=True, steps=10, total_disp=0.01,
              critical_bstrain=1.0, tol_iter=1e-5, max_iter=30) -> Case:
    """Config 1 (ex1_isoelasticity_2d_hex): hexagonal plate, bottom edge fixed, top edge pulled
    in y by total_disp over `steps` equal steps.  Groups as ex1_isoelasticity_2d_hex.cpp:72-81."""
    box = [0.0, size, 0.0, size, 0.0, 1.0]
    xyz = _gen(L.LatticeType.Hexagon2D, radius, box)
    top = np.nonzero(xyz[:, 1] > box[3] - 2 * radius)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 1] < box[2] + 2 * radius)[0].astype(np.int32)
    types = np.zeros(len(xyz), np.int32)
    types[top] = 1
    types[bot] = 2
    mat = L.Material(plane_stress=plane_stress, E=E, mu=mu, critical_bstrain=critical_bstrain)
    dstep = total_disp / steps
    st = [([("bottom", "x", 0.0), ("bottom", "y", 0.0), ("top", "y", dstep)], []) for _ in range(steps)]
    return Case(f"hex2d_{size:g}mm_r{radius:g}", L.LatticeType.Hexagon2D, radius, box, xyz, L.ParticleType.Elastic,
                mat, types, {"top": top, "bottom": bot}, st, tol_iter=tol_iter, max_iter=max_iter)


def sc_cube(size=20.0, radius=0.2, E=2e5, mu=0.25, steps=20, total_disp=0.02, tol_iter=1e-5, max_iter=30,
            ptype=L.ParticleType.Elastic, j2=None, lattice=L.LatticeType.SimpleCubic3D) -> Case:
    """Config 2 (ex1_isoelasticity_3d_sc): simple-cubic cube, bottom face fixed in z, one bottom
    corner pinned in x and y, and a second bottom corner fixed in y so the rotation about z is
    removed (a single pinned corner leaves K singular); top face pulled in z.  `lattice` may be
    BCC3D for the same cube on a body-centred cubic lattice."""
    box = [0.0, size, 0.0, size, 0.0, size]
    xyz = _gen(lattice, radius, box)
    top = np.nonzero(xyz[:, 2] > box[5] - 2 * radius)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 2] < box[4] + 2 * radius)[0].astype(np.int32)
    zb = xyz[bot]
    c0 = bot[np.lexsort((zb[:, 2], zb[:, 1], zb[:, 0]))[0]]              # min x, then min y
    c1 = bot[np.lexsort((zb[:, 2], zb[:, 1], -zb[:, 0]))[0]]             # max x, then min y
    types = np.zeros(len(xyz), np.int32)
    types[top] = 1
    types[bot] = 2
    mat = L.Material(plane_stress=False, E=E, mu=mu)
    if j2 is not None:
        mat.sigmay, mat.xi, mat.H, mat.A = j2
    dstep = total_disp / steps
    groups = {"top": top, "bottom": bot, "corner0": np.array([c0], np.int32), "corner1": np.array([c1], np.int32)}
    st = [([("bottom", "z", 0.0), ("corner0", "x", 0.0), ("corner0", "y", 0.0), ("corner1", "y", 0.0),
            ("top", "z", dstep)], []) for _ in range(steps)]
    tag = "sc3d" if lattice == L.LatticeType.SimpleCubic3D else "bcc3d"
    return Case(f"{tag}_{size:g}mm_r{radius:g}", L.LatticeType(lattice), radius, box, xyz, ptype, mat, types,
                groups, st, tol_iter=tol_iter, max_iter=max_iter)


def fcc_bar(size=(4.0, 4.0, 8.0), radius=0.2, E=110e3, mu=0.34, steps=10, strain=0.01, seed=7,
            j2=(60.0 * 3.06, 0.0, 500.0, 0.0), tol_iter=1e-5, max_iter=30) -> Case:
    """Config 3: FCC single crystal in J2 plasticity (the reference has no crystal plasticity),
    Bunge orientation from a seeded uniform rotation, tension to `strain` in `steps` steps.
    sigma_y = CRSS 60 MPa x Taylor factor 3.06."""
    rng = np.random.default_rng(seed)
    phi1, Phi, phi2 = 2 * math.pi * rng.random(), math.acos(1 - 2 * rng.random()), 2 * math.pi * rng.random()
    box = [0.0, size[0], 0.0, size[1], 0.0, size[2]]
    euler = (2, (phi1, Phi, phi2))
    xyz = _gen(L.LatticeType.FCC3D, radius, box, euler)
    top = np.nonzero(xyz[:, 2] > box[5] - 2 * radius)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 2] < box[4] + 2 * radius)[0].astype(np.int32)
    zb = xyz[bot]
    c0 = bot[np.lexsort((zb[:, 2], zb[:, 1], zb[:, 0]))[0]]
    c1 = bot[np.lexsort((zb[:, 2], zb[:, 1], -zb[:, 0]))[0]]
    types = np.zeros(len(xyz), np.int32)
    mat = L.Material(plane_stress=False, E=E, mu=mu)
    mat.sigmay, mat.xi, mat.H, mat.A = j2
    dstep = strain * size[2] / steps
    groups = {"top": top, "bottom": bot, "corner0": np.array([c0], np.int32), "corner1": np.array([c1], np.int32)}
    st = [([("bottom", "z", 0.0), ("corner0", "x", 0.0), ("corner0", "y", 0.0), ("corner1", "y", 0.0),
            ("top", "z", dstep)], []) for _ in range(steps)]
    return Case(f"fcc3d_j2_r{radius:g}", L.LatticeType.FCC3D, radius, box, xyz, L.ParticleType.J2Plasticity, mat,
                types, groups, st, tol_iter=tol_iter, max_iter=max_iter, euler=euler)


def fcc_cubic_cube(size=2.8, radius=0.244948964611159, C11=108e3, C12=61e3, C44=29e3, steps=2, total_disp=0.002,
                   critical_bstrain=1.0, tol_iter=1e-9, max_iter=30) -> Case:
    """An FCC cube of elastic particles with cubic elastic constants, as
    examples/ex3_singlecrystal_3d_fcc.cpp sets them (setParticleProperty's (C11, C12, C44) overload,
    particle_elastic.h:110-140; its radius and constants): bottom face fixed in z with two corners
    pinned, top face moved in z."""
    c = sc_cube(size=size, radius=radius, steps=steps, total_disp=total_disp, tol_iter=tol_iter, max_iter=max_iter,
                lattice=L.LatticeType.FCC3D)
    c.name = f"fcc_cubic_{size:g}mm"
    c.material.C11, c.material.C12, c.material.C44 = C11, C12, C44
    c.material.critical_bstrain = critical_bstrain
    return c


def notched_plate(size=4.0, radius=0.1, crack=0.3, E=69e3, mu=0.3, critical_bstrain=2e-3, steps=40,
                  total_disp=None, tol_iter=1e-5, max_iter=30) -> Case:
    """Single-edge-notched hexagonal plate with brittle bonds, pulled in y.  The pre-crack is a
    straight slit from the left edge, ``crack`` x the width long, between the two particle rows
    nearest mid-height; the bonds crossing it are left out of the bond lists (the bond-exclusion
    of geometry/geo1_CT_configuration.cpp:79-134, read back through Assembly::readBond)."""
    box = [0.0, size, 0.0, size, 0.0, 1.0]
    xyz = _gen(L.LatticeType.Hexagon2D, radius, box)
    top = np.nonzero(xyz[:, 1] > box[3] - 2 * radius)[0].astype(np.int32)
    bot = np.nonzero(xyz[:, 1] < box[2] + 2 * radius)[0].astype(np.int32)
    types = np.zeros(len(xyz), np.int32)
    types[top] = 1
    types[bot] = 2
    mat = L.Material(plane_stress=True, E=E, mu=mu, critical_bstrain=critical_bstrain)
    if total_disp is None:
        total_disp = 3.0 * critical_bstrain * size
    dstep = total_disp / steps
    st = [([("bottom", "x", 0.0), ("bottom", "y", 0.0), ("top", "y", dstep)], []) for _ in range(steps)]
    c = Case(f"sen_hex_{size:g}mm", L.LatticeType.Hexagon2D, radius, box, xyz, L.ParticleType.Elastic, mat, types,
             {"top": top, "bottom": bot}, st, tol_iter=tol_iter, max_iter=max_iter)
    ys = np.unique(np.round(xyz[:, 1], 9))
    k = int(np.searchsorted(ys, 0.5 * size)) - 1
    k = min(max(k, 0), len(ys) - 2)
    y_slit = 0.5 * (ys[k] + ys[k + 1])
    c.bonds = bond_lists(xyz, L.UnitCell(L.LatticeType.Hexagon2D, radius),
                         slit_exclusion(xyz, y_slit, box[0] - 1.0, box[0] + crack * size))
    c.meta["crack"] = (crack * size, y_slit)
    return c


def cantilever_beam(radius=0.12, length=30.0, depth=10.0, force=2.0, E=69e3, mu=0.33, tol_iter=1e-5,
                    max_iter=30) -> Case:
    """The known-answer case of examples/ex7_convergence_beam.cpp: a plane-strain hexagonal beam,
    box {0, length, -depth/2, depth/2}, its right edge (x > xmax - EPS) fixed in x and y and its
    left edge (x < xmin + EPS) loaded by `force` in y, shared by its particles, in one step.  The
    example's nonlocal search (cutoff 1.5 x nonlocal_L = EPS) finds each particle alone and the
    undamaged type 4 matches no particle; neither changes an elastic solve."""
    box = [0.0, length, -depth / 2, depth / 2, 0.0, 1.0]
    xyz = _gen(L.LatticeType.Hexagon2D, radius, box)
    eps = 1e-6  # EPS, include/lpm.h:41
    xmin, xmax = float(xyz[:, 0].min()), float(xyz[:, 0].max())
    left = np.nonzero(xyz[:, 0] < xmin + eps)[0].astype(np.int32)
    right = np.nonzero(xyz[:, 0] > xmax - eps)[0].astype(np.int32)
    types = np.zeros(len(xyz), np.int32)
    types[left] = 2
    types[right] = 1
    mat = L.Material(plane_stress=False, E=E, mu=mu, critical_bstrain=1.0, nonlocal_L=eps)
    st = [([("right", "x", 0.0), ("right", "y", 0.0)], [("left", 0.0, force, 0.0)])]
    c = Case(f"beam_{length:g}x{depth:g}_r{radius:g}", L.LatticeType.Hexagon2D, radius, box, xyz,
             L.ParticleType.Elastic, mat, types, {"left": left, "right": right}, st, undamaged_type=4,
             tol_iter=tol_iter, max_iter=max_iter)
    c.nonlocal_cutoff_ratio = 1.5
    c.meta.update({"length": box[1] - box[0], "depth": box[3] - box[2], "force": force})
    return c


def edamage_plate(size=2.4, radius=0.1, E=69e3, mu=0.3, steps=4, total_disp=0.008, k0=0.02, k1=0.5,
                  damage_threshold=0.9, nonlocal_L=0.3, cutoff_ratio=1.5, tol_iter=1e-9, max_iter=30,
                  undamaged_band=0.0) -> Case:
    """Hexagonal plate of ParticleElasticDamage particles (include/particle_elastic_damage.h) with
    the nonlocal damage of SolverStatic::updateStaticDamage (solver_static.h:32-62): the bottom edge
    fixed, the top edge pulled in y (the groups of ex1_isoelasticity_2d_hex).  Damage grows once
    the strain energy density passes k0 + k1 D; the local rates are averaged over the neighbours
    within cutoff_ratio x nonlocal_L (Assembly::searchNonlocalNeighbors, assembly.h:118-130).
    undamaged_band > 0 gives the particles within that distance of the top and bottom edges,
    outside the loaded edge groups, type 3 and makes 3 the undamaged type: they take no damage
    and are left out of the averaging (solver_static.h:37-57)."""
    c = hex_plate(size=size, radius=radius, E=E, mu=mu, steps=steps, total_disp=total_disp, tol_iter=tol_iter,
                  max_iter=max_iter)
    c.name = f"edamage_hex_{size:g}mm"
    c.ptype = L.ParticleType.ElasticDamage
    if undamaged_band > 0:
        y = c.xyz[:, 1]
        far = (y > y.max() - undamaged_band) | (y < y.min() + undamaged_band)
        c.types = c.types.copy()
        c.types[far & (c.types == 0)] = 3
        c.undamaged_type = 3
    c.material.k0, c.material.k1, c.material.damage_threshold = k0, k1, damage_threshold
    c.material.nonlocal_L = nonlocal_L
    c.nonlocal_cutoff_ratio = cutoff_ratio
    c.meta.update({"k0": k0, "k1": k1, "damage_threshold": damage_threshold, "nonlocal_L": nonlocal_L,
                   "cutoff_ratio": cutoff_ratio})
    return c


def fatigue_plate(size=2.4, radius=0.1, E=69e3, mu=0.3, amplitude=0.004, cycles=8, n_interval=2, tau=0.5,
                  tmode="linear", A=15.0, B=2.833, d=0.5, damage_threshold=1.0, fatigue_limit_ratio=1.108,
                  nonlocal_L=0.3, cutoff_ratio=1.5, tol_iter=1e-9, max_iter=30, load_type="uniaxial_disp",
                  undamaged_band=0.0) -> Case:
    """Hexagonal plate of ParticleFatigueHCF particles (include/particle_fatigue_hcf.h) under the
    constant-amplitude displacement cycles of SolverFatigue (include/solver_fatigue.h) with the
    LoadUniaxialDisp cycle (include/load_step_fatigue.h:39-50): left edge fixed in x, bottom edge
    in y, top edge moved in y.  One static step first (solveProblemStatic at f_min = 0, which
    sets the constraints, as ex5_isoelasticity_2d_fatigue.cpp does before its cycles), then the
    spectrum 0, amplitude, 0, amplitude, ..., 0 of `cycles` cycles.  load_type "uniaxial_force"
    takes the LoadUniaxialForce cycle instead (load_step_fatigue.h:23-36): the top edge pulled by a
    force of `amplitude` N shared by its particles, and "ct_force" the LoadCTForce cycle (the middle
    row held in y, the top and bottom edges held in x and pulled apart by +/- `amplitude` N).
    undamaged_band > 0 gives the particles within that distance of the top and bottom edges type 3,
    the undamaged type, outside the loaded edge groups (types 1 and 2), as
    examples/ex5_isoelasticity_2d_fatigue.cpp types the grips of its specimen.  Each simulated cycle stands
    for dN/dt = (int)(1 / tau) real cycles (TimeMapMode::Linear, solver_fatigue.h:60-63); the
    damage rate per cycle is A * pow(largest energy, B) * pow(energy range, d), averaged over the
    nonlocal neighbours within cutoff_ratio x nonlocal_L."""
    c = hex_plate(size=size, radius=radius, E=E, mu=mu, steps=1, total_disp=0.0, tol_iter=tol_iter,
                  max_iter=max_iter)
    c.name = f"fatigue_hex_{size:g}mm"
    c.ptype = L.ParticleType.FatigueHCF
    x = c.xyz[:, 0]
    c.groups["left"] = np.nonzero(x < x.min() + 1.5 * radius)[0].astype(np.int32)
    if load_type == "uniaxial_force":  # the top edge stays free in y: the force moves it
        c.steps = [([("left", "x", 0.0), ("bottom", "y", 0.0)], [])]
    elif load_type == "ct_force":  # LoadCTForce (load_step_fatigue.h:71-87): mid row held in y,
        y = c.xyz[:, 1]             # top and bottom edges held in x and pulled apart in y
        ymid = 0.5 * (y.min() + y.max())
        c.groups["mid"] = np.nonzero(np.abs(y - ymid) < radius)[0].astype(np.int32)
        c.steps = [([("mid", "y", 0.0), ("top", "x", 0.0), ("bottom", "x", 0.0)], [])]
    else:
        c.steps = [([("left", "x", 0.0), ("top", "y", 0.0), ("bottom", "y", 0.0)], [])]
    if undamaged_band > 0:
        y = c.xyz[:, 1]
        far = (y > y.max() - undamaged_band) | (y < y.min() + undamaged_band)
        c.types = c.types.copy()
        c.types[far & (c.types == 0)] = 3
        c.undamaged_type = 3
    m = c.material
    m.fatigue_A, m.fatigue_B, m.fatigue_d = A, B, d
    m.damage_threshold, m.fatigue_limit_ratio, m.nonlocal_L = damage_threshold, fatigue_limit_ratio, nonlocal_L
    c.nonlocal_cutoff_ratio = cutoff_ratio
    spectrum = [0.0] + [v for _ in range(cycles) for v in (amplitude, 0.0)]
    groups = ["mid", "top", "bottom"] if load_type == "ct_force" else ["left", "top", "bottom"]
    c.meta["fatigue"] = {"load_type": load_type, "n_interval": n_interval, "tmode": tmode, "tau": tau,
                         "spectrum": spectrum, "groups": groups}
    return c


def fatigue_cube(size=2.0, radius=0.2, E=69e3, mu=0.3, amplitude=0.004, cycles=4, n_interval=2, tau=0.5,
                 A=15.0, B=2.833, d=0.5, damage_threshold=1.0, nonlocal_L=0.6, cutoff_ratio=1.5, tol_iter=1e-9,
                 max_iter=30) -> Case:
    """A simple-cubic cube of fatigue HCF particles under the LoadDogBoneDisp cycle
    (load_step_fatigue.h:53-69), as examples/ex5_isoelasticity_3d_fatigue.cpp loads its specimen:
    the top layer (largest y) moved in y and held in x and z, the bottom layer held in x, y and z.
    One static step at zero load, then `cycles` cycles of the spectrum 0, amplitude, 0, ..."""
    c = sc_cube(size=size, radius=radius, E=E, mu=mu, steps=1, total_disp=0.0, tol_iter=tol_iter, max_iter=max_iter)
    c.name = f"fatigue_sc_{size:g}mm"
    c.ptype = L.ParticleType.FatigueHCF
    y = c.xyz[:, 1]
    c.groups = {"top": np.nonzero(y > y.max() - radius)[0].astype(np.int32),
                "bottom": np.nonzero(y < y.min() + radius)[0].astype(np.int32)}
    c.types = np.zeros(c.n, np.int32)
    c.steps = [([("top", "x", 0.0), ("top", "y", 0.0), ("top", "z", 0.0), ("bottom", "x", 0.0),
                 ("bottom", "y", 0.0), ("bottom", "z", 0.0)], [])]
    m = c.material
    m.fatigue_A, m.fatigue_B, m.fatigue_d = A, B, d
    m.damage_threshold, m.nonlocal_L = damage_threshold, nonlocal_L
    c.nonlocal_cutoff_ratio = cutoff_ratio
    spectrum = [0.0] + [v for _ in range(cycles) for v in (amplitude, 0.0)]
    c.meta["fatigue"] = {"load_type": "dogbone_disp", "n_interval": n_interval, "tmode": "linear", "tau": tau,
                         "spectrum": spectrum, "groups": ["top", "bottom"]}
    return c


def batched_notched_plates(count=64, seed=20240604, steps=40, radius=0.1, side=(4.0, 25.0), crack=(0.2, 0.5),
                           E=(60e3, 120e3), critical_bstrain=(1e-3, 3e-3), opening=0.45, crack_ref=1.5,
                           tol_iter=1e-5, max_iter=30) -> List[Case]:
    """Batched 2D damage workload: ``count`` single-edge-notched hexagonal plates of uneven size.
    Per plate (seeded): side L log-uniform in ``side`` mm at radius 0.1 mm, slit length a uniform
    in ``crack`` x L, E uniform in ``E`` MPa, nu = 0.3, critical bond stretch c uniform in
    ``critical_bstrain``.  Mode I: bottom edge fixed, top edge pulled in y in ``steps`` equal
    steps to a total opening of ``opening`` x c x L x min(1, sqrt(crack_ref / a)).
    The square-root factor keeps the slit tip's loading (stress intensity ~ strain x sqrt(a))
    about equal across sizes: the tip breaks bonds and the crack starts to grow in every plate,
    but does not run through.  Larger loads (checked with the oracle and the plain GPU path)
    leave particles hanging on single bonds or split the plate; K is then singular, CG runs to
    its iteration cap and the reference's own path ends in NaN."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        L = float(np.exp(rng.uniform(np.log(side[0]), np.log(side[1]))))
        L = round(L / (2 * radius)) * 2 * radius
        a = float(rng.uniform(*crack))
        e = float(rng.uniform(*E))
        cs = float(rng.uniform(*critical_bstrain))
        scale = min(1.0, math.sqrt(crack_ref / (a * L)))
        c = notched_plate(size=L, radius=radius, crack=a, E=e, mu=0.3, critical_bstrain=cs, steps=steps,
                          total_disp=opening * cs * L * scale, tol_iter=tol_iter, max_iter=max_iter)
        c.name = f"sen{k:02d}_L{L:.1f}"
        c.meta.update({"seed": seed, "index": k, "side": L, "crack_ratio": a, "E": e, "critical_bstrain": cs,
                       "opening_scale": scale})
        out.append(c)
    return out


def serving_requests(count=16, seed=20240605, rate=200.0, n_range=(5e3, 5e5), steps_range=(5, 50), strain=1e-3,
                     j2=(200.0, 0.0, 38714.0, 10.0)):
    """Serving stream: `count` requests with Poisson arrivals (seeded, mean `rate` per second).
    Per request: lattice hex-2D, SC-3D or BCC-3D (equally likely), particle count log-uniform in
    `n_range` (the specimen side is chosen to give about that count), E uniform 50-250 GPa, nu
    uniform 0.2-0.35, a monotone path of 5-50 equal steps to `strain` total strain, elastic or
    (3D lattices, half of them) J2 plasticity.  Returns [(arrival seconds, Case)]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for k in range(count):
        t += float(rng.exponential(1.0 / rate))
        lat = int(rng.integers(0, 3))
        n = float(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        E = float(rng.uniform(50e3, 250e3))
        mu = float(rng.uniform(0.2, 0.35))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        plastic = bool(rng.random() < 0.5)
        if lat == 0:
            side = round(math.sqrt(n / 29.0), 1)  # hexagonal plate at r = 0.1: ~29 particles per mm^2
            c = hex_plate(size=side, radius=0.1, E=E, mu=mu, steps=steps, total_disp=strain * side)
        else:
            lattice = L.LatticeType.SimpleCubic3D if lat == 1 else L.LatticeType.BCC3D
            per_edge = n ** (1.0 / 3.0) if lat == 1 else (n / 2.0) ** (1.0 / 3.0)
            cellw = 0.4 if lat == 1 else 4 * 0.2 / math.sqrt(3.0)
            side = round(per_edge * cellw, 1)
            c = sc_cube(size=side, radius=0.2, E=E, mu=mu, steps=steps, total_disp=strain * side, lattice=lattice,
                        ptype=L.ParticleType.J2Plasticity if plastic else L.ParticleType.Elastic,
                        j2=j2 if plastic else None)
        c.name = f"req{k:02d}_{c.name}"
        c.meta.update({"arrival": t, "seed": seed, "index": k})
        out.append((t, c))
    return out
