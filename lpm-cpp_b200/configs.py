"""Synthetic LPM workloads: lattices from the reference's generators, the boundary groups and
load paths of the reference examples, sized as the benchmark configurations.

A ``Case`` is plain data (coordinates, particle types, material, groups, load steps) so the
same problem can be handed to the device solver and to the CPU oracle.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Dict, List, Tuple

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
        return a


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
            ptype=L.ParticleType.Elastic, j2=None) -> Case:
    """Config 2 (ex1_isoelasticity_3d_sc): simple-cubic cube, bottom face fixed in z, one bottom
    corner pinned in x and y, and a second bottom corner fixed in y so the rotation about z is
    removed (a single pinned corner leaves K singular); top face pulled in z."""
    box = [0.0, size, 0.0, size, 0.0, size]
    xyz = _gen(L.LatticeType.SimpleCubic3D, radius, box)
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
    return Case(f"sc3d_{size:g}mm_r{radius:g}", L.LatticeType.SimpleCubic3D, radius, box, xyz, ptype, mat, types,
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


def notched_plate(size=4.0, radius=0.1, crack=0.3, E=69e3, mu=0.3, critical_bstrain=2e-3, steps=40,
                  total_disp=None, tol_iter=1e-5, max_iter=30) -> Case:
    """Config 4 member: single-edge-notched hexagonal plate, brittle bonds.  The pre-crack is a
    straight slit from the left edge at mid-height, made by leaving out the bonds that cross
    it (the bond-exclusion pattern of geometry/geo1_CT_configuration.cpp:79-134), realised here
    by giving the particles on the two faces of the slit broken bonds across it."""
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
    c.meta["crack"] = (crack * size, 0.5 * size)
    return c
