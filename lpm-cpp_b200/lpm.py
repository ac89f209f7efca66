"""Host-side mirror of the LPM-CPP interface for the implicit quasi-static step, over the C ABI
of liblpmgpu.so (include/lpmgpu.h).

The names follow the reference so an example's ``run()`` reads the same:
``UnitCell``, ``createRMatrix``, ``createPlateHEX2D`` / ``createPlateSQ2D`` /
``createCuboidSC3D`` / ``createCuboidFCC3D`` (include/utilities.h), ``Assembly``
(include/assembly.h), ``LoadStep`` / ``DispBC`` / ``ForceBC`` (include/load_step.h,
include/boundary.h) and ``SolverStatic`` with ``solveProblem(load, start_index)``
(include/solver_static.h).  The solver runs on the GPU only: without liblpmgpu.so or a CUDA
device the constructors raise; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes as C
import enum
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblpmgpu.so")


class LatticeType(enum.IntEnum):
    Square2D = 0
    Hexagon2D = 1
    SimpleCubic3D = 2
    FCC3D = 3
    BCC3D = 4


class ParticleType(enum.IntEnum):
    Elastic = 0
    ElasticDamage = 1
    J2Plasticity = 2
    FatigueHCF = 3


class LoadMode(enum.IntEnum):
    Relative = 0
    Absolute = 1


class SolverMode(enum.IntEnum):
    CG = 0
    PARDISO = 1


class StiffnessMode(enum.IntEnum):
    Analytical = 0
    FiniteDifference = 1


class Precision(enum.IntEnum):
    FP64 = 0
    MIXED = 1


STATUS = {0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory",
          4: "Newton iteration did not converge", 5: "CG reached its iteration cap",
          6: "device wait timed out", 7: "unsupported particle topology", 8: "HBM budget exceeded",
          9: "load step halved too many times", 10: "result not ready", 11: "no CUDA device",
          12: "stiffness not positive definite", 13: "CG broke down (p.Ap == 0)"}
OK, ERR_NEWTON, ERR_CUTS, ERR_NOT_READY = 0, 4, 9, 10
ERR_CG_MAXIT, ERR_TIMEOUT, ERR_CG_BREAKDOWN = 5, 6, 13


class LpmGpuError(RuntimeError):
    def __init__(self, status: int, where: str):
        msg = STATUS.get(status, "unknown")
        detail = ""
        if _lib is not None:
            detail = _lib.lpmgpu_last_error().decode(errors="replace")
        super().__init__(f"{where}: {msg} ({status}){': ' + detail if detail else ''}")
        self.status = status


# ---------------------------------------------------------------------------- C ABI structs
class Desc(C.Structure):
    _fields_ = [
        ("lattice", C.c_int32), ("ptype", C.c_int32), ("n", C.c_int32),
        ("xyz", C.POINTER(C.c_double)), ("type", C.POINTER(C.c_int32)),
        ("radius", C.c_double), ("plane_stress", C.c_int32),
        ("E", C.c_double), ("mu", C.c_double), ("critical_bstrain", C.c_double),
        ("sigmay", C.c_double), ("xi", C.c_double), ("H", C.c_double), ("A", C.c_double),
        ("nonlocal_L", C.c_double), ("undamaged_type", C.c_int32), ("max_iter", C.c_int32),
        ("tol_iter", C.c_double), ("cg_rtol", C.c_double), ("cg_atol", C.c_double),
        ("cg_maxit", C.c_int64), ("precision", C.c_int32), ("device", C.c_int32),
        ("bond_nb0", C.POINTER(C.c_int32)), ("bond_nb1", C.POINTER(C.c_int32)), ("bond_p2", C.POINTER(C.c_int32)),
        ("bond_kn", C.POINTER(C.c_double)), ("bond_tv", C.POINTER(C.c_double)),
        ("bond_damage", C.POINTER(C.c_double)), ("tangent", C.c_int32),
        ("nonlocal_cutoff_ratio", C.c_double), ("k0", C.c_double), ("k1", C.c_double),
        ("comp_tensile_ratio", C.c_double), ("damage_threshold", C.c_double),
        ("fatigue_A", C.c_double), ("fatigue_B", C.c_double), ("fatigue_d", C.c_double),
        ("fatigue_limit_ratio", C.c_double),
        ("nonlocal_count", C.POINTER(C.c_int32)), ("nonlocal_ids", C.POINTER(C.c_int32)),
        ("direct", C.c_int32),
        ("C11", C.c_double), ("C12", C.c_double), ("C44", C.c_double),
    ]


class CDispBC(C.Structure):
    _fields_ = [("ids", C.POINTER(C.c_int32)), ("count", C.c_int32), ("flag", C.c_int32), ("step", C.c_double)]


class CForceBC(C.Structure):
    _fields_ = [("ids", C.POINTER(C.c_int32)), ("count", C.c_int32),
                ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double)]


class CLoadStep(C.Structure):
    _fields_ = [("disp", C.POINTER(CDispBC)), ("ndisp", C.c_int32),
                ("force", C.POINTER(CForceBC)), ("nforce", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("converged", C.c_int32), ("newton_solves", C.c_int32), ("cuts", C.c_int32),
                ("damage_iters", C.c_int32), ("cg_iters", C.c_int64), ("cg_maxit_hits", C.c_int64),
                ("refinements", C.c_int32), ("reaction_norm", C.c_double), ("residual_norm", C.c_double),
                ("seconds", C.c_double), ("direct_solves", C.c_int32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Counters(C.Structure):
    _fields_ = [("kernel_launches", C.c_int64), ("cg_launches", C.c_int64), ("cg_iters", C.c_int64),
                ("cg_kernel_seconds", C.c_double), ("assembly_seconds", C.c_double), ("force_seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Sizes(C.Structure):
    _fields_ = [("n", C.c_int32), ("dim", C.c_int32), ("nbonds", C.c_int64), ("nnzb", C.c_int64),
                ("nnz_upper", C.c_int64), ("max_bonds", C.c_int32), ("max_conns", C.c_int32),
                ("device_bytes", C.c_int64)]


class MemberInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("steps_done", C.c_int32), ("nsteps", C.c_int32),
                ("total", Stats), ("dof_iters", C.c_int64), ("seconds", C.c_double)]


class RequestInfo(C.Structure):
    _fields_ = [("state", C.c_int32), ("status", C.c_int32), ("n", C.c_int32), ("steps_done", C.c_int32),
                ("nsteps", C.c_int32), ("total", Stats), ("dof_iters", C.c_int64), ("device_bytes", C.c_int64),
                ("t_submit", C.c_double), ("t_start", C.c_double), ("t_done", C.c_double)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "total"}
        d["total"] = self.total.as_dict()
        return d


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("queued", C.c_int64), ("running", C.c_int64), ("done", C.c_int64),
                ("failed", C.c_int64), ("rounds", C.c_int64), ("bytes_in_use", C.c_int64),
                ("bytes_budget", C.c_int64), ("peak_bytes", C.c_int64), ("worker_status", C.c_int32),
                ("pad", C.c_int32), ("latency_p50", C.c_double), ("latency_p99", C.c_double),
                ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class TuneResult(C.Structure):
    _fields_ = [("precision", C.c_int32), ("grid_default", C.c_int32), ("grid_chosen", C.c_int32),
                ("ncandidates", C.c_int32), ("grid", C.c_int32 * 8), ("us_per_iter", C.c_double * 8)]

    def as_dict(self):
        k = self.ncandidates
        return {"precision": self.precision, "grid_default": self.grid_default, "grid_chosen": self.grid_chosen,
                "candidates": list(self.grid[:k]), "us_per_iter": list(self.us_per_iter[:k])}


class BatchStats(C.Structure):
    _fields_ = [("rounds", C.c_int64), ("cg_launches", C.c_int64), ("members_done", C.c_int64),
                ("members_failed", C.c_int64), ("cg_iters", C.c_int64), ("dof_iters", C.c_int64),
                ("seconds", C.c_double), ("cg_kernel_seconds", C.c_double), ("fp32_kernel", C.c_int32),
                ("fp32_kernel_small", C.c_int32), ("fp32_tuning", C.c_int32), ("pad", C.c_int32),
                ("solo_solves", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# every symbol declared in include/lpmgpu.h
EXPORTS = [
    "lpmgpu_version", "lpmgpu_status_string", "lpmgpu_last_error", "lpmgpu_generate_lattice",
    "lpmgpu_create", "lpmgpu_destroy", "lpmgpu_get_sizes", "lpmgpu_get_topology",
    "lpmgpu_update_force_state", "lpmgpu_update_state_var", "lpmgpu_update_rr", "lpmgpu_assemble",
    "lpmgpu_export_ref_csr", "lpmgpu_solve_linear", "lpmgpu_apply_load_step",
    "lpmgpu_solve_problem_step", "lpmgpu_solve_load_step", "lpmgpu_store_state", "lpmgpu_reset_state",
    "lpmgpu_fatigue_solve_step", "lpmgpu_fatigue_static_step", "lpmgpu_fatigue_update_damage", "lpmgpu_fatigue_cycle",
    "lpmgpu_read_state", "lpmgpu_read_residual", "lpmgpu_set_xyz", "lpmgpu_get_phase_times",
    "lpmgpu_get_counters", "lpmgpu_get_stream", "lpmgpu_cg_bsr_noalloc", "lpmgpu_autotune", "lpmgpu_set_cg_grid",
    "lpmgpu_set_wait_limit_ns", "lpmgpu_set_assembly_exact",
    "lpmgpu_solve_direct", "lpmgpu_band_order", "lpmgpu_get_nonlocal",
    "lpmgpu_format_dump", "lpmgpu_dump_write", "lpmgpu_dump_flush",
    "lpmgpu_batch_create", "lpmgpu_batch_destroy", "lpmgpu_batch_add", "lpmgpu_batch_add_fatigue",
    "lpmgpu_batch_round", "lpmgpu_batch_run",
    "lpmgpu_batch_member", "lpmgpu_batch_member_steps", "lpmgpu_batch_remove", "lpmgpu_batch_get_stats",
    "lpmgpu_batch_set_slice", "lpmgpu_batch_set_lanes", "lpmgpu_batch_set_solo_bytes",
    "lpmgpu_estimate_bytes", "lpmgpu_server_create", "lpmgpu_server_destroy", "lpmgpu_server_set_slice", "lpmgpu_server_set_lanes", "lpmgpu_server_set_solo_bytes", "lpmgpu_server_submit",
    "lpmgpu_server_submit_fatigue",
    "lpmgpu_server_poll", "lpmgpu_server_wait", "lpmgpu_server_result", "lpmgpu_server_get_stats",
]


def lib():
    """Loads liblpmgpu.so (built by lpm-cpp_b200/build.py); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'`")
    L = C.CDLL(LIB_PATH)
    vp, dp, ip, lp = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int32), C.POINTER(C.c_int64)
    sig = {
        "lpmgpu_version": (C.c_char_p, []),
        "lpmgpu_status_string": (C.c_char_p, [C.c_int32]),
        "lpmgpu_last_error": (C.c_char_p, []),
        "lpmgpu_generate_lattice": (C.c_int32, [C.c_int32, C.c_double, dp, C.c_int32, dp, dp, C.c_int64, lp]),
        "lpmgpu_create": (C.c_int32, [C.POINTER(Desc), C.POINTER(vp)]),
        "lpmgpu_destroy": (C.c_int32, [vp]),
        "lpmgpu_get_sizes": (C.c_int32, [vp, C.POINTER(Sizes)]),
        "lpmgpu_get_topology": (C.c_int32, [vp, ip, ip, ip, ip, ip, ip]),
        "lpmgpu_update_force_state": (C.c_int32, [vp]),
        "lpmgpu_update_state_var": (C.c_int32, [vp]),
        "lpmgpu_update_rr": (C.c_int32, [vp, dp]),
        "lpmgpu_assemble": (C.c_int32, [vp, C.c_int32]),
        "lpmgpu_export_ref_csr": (C.c_int32, [vp, lp, lp, lp, dp]),
        "lpmgpu_solve_linear": (C.c_int32, [vp, dp, C.POINTER(Stats)]),
        "lpmgpu_apply_load_step": (C.c_int32, [vp, C.POINTER(CLoadStep)]),
        "lpmgpu_solve_problem_step": (C.c_int32, [vp, C.POINTER(CLoadStep), C.POINTER(Stats)]),
        "lpmgpu_solve_load_step": (C.c_int32, [vp, C.POINTER(CLoadStep), C.POINTER(Stats)]),
        "lpmgpu_fatigue_solve_step": (C.c_int32, [vp, C.POINTER(CLoadStep), C.POINTER(Stats)]),
        "lpmgpu_fatigue_static_step": (C.c_int32, [vp, C.POINTER(CLoadStep), C.POINTER(Stats)]),
        "lpmgpu_fatigue_update_damage": (C.c_int32, [vp, C.c_double, ip]),
        "lpmgpu_fatigue_cycle": (C.c_int32, [vp, C.POINTER(CLoadStep), C.c_int32, C.c_double, C.POINTER(Stats), ip]),
        "lpmgpu_store_state": (C.c_int32, [vp]),
        "lpmgpu_reset_state": (C.c_int32, [vp]),
        "lpmgpu_read_state": (C.c_int32, [vp, dp, dp, dp, dp, dp, dp, dp]),
        "lpmgpu_read_residual": (C.c_int32, [vp, dp]),
        "lpmgpu_set_xyz": (C.c_int32, [vp, dp]),
        "lpmgpu_get_phase_times": (C.c_int32, [vp, dp]),
        "lpmgpu_get_counters": (C.c_int32, [vp, C.POINTER(Counters)]),
        "lpmgpu_get_stream": (C.c_int32, [vp, C.POINTER(vp)]),
        "lpmgpu_format_dump": (C.c_int32, [C.c_char_p, C.c_int32, C.c_int32, ip, dp, dp, dp, dp, dp, dp, dp,
                                           C.c_int32, C.c_int32]),
        "lpmgpu_dump_write": (C.c_int32, [vp, C.c_char_p, C.c_int32, dp, C.c_int32, C.c_int32]),
        "lpmgpu_dump_flush": (C.c_int32, [vp]),
        "lpmgpu_autotune": (C.c_int32, [vp, C.c_int32, C.POINTER(TuneResult)]),
        "lpmgpu_solve_direct": (C.c_int32, [vp, dp, C.POINTER(Stats)]),
        "lpmgpu_band_order": (C.c_int32, [C.c_int32, ip, ip, ip, lp]),
        "lpmgpu_get_nonlocal": (C.c_int32, [vp, ip, ip, lp]),
        "lpmgpu_set_cg_grid": (C.c_int32, [vp, C.c_int32]),
        "lpmgpu_set_wait_limit_ns": (C.c_int32, [vp, C.c_int64]),
        "lpmgpu_set_assembly_exact": (C.c_int32, [vp, C.c_int32]),
        "lpmgpu_cg_bsr_noalloc": (C.c_int32, [C.c_int32, C.c_int32, vp, vp, vp, vp, vp, C.c_double, C.c_double,
                                              C.c_int64, vp, C.POINTER(C.c_int64)]),
        "lpmgpu_batch_create": (C.c_int32, [C.c_int32, C.POINTER(vp)]),
        "lpmgpu_batch_destroy": (C.c_int32, [vp]),
        "lpmgpu_batch_add": (C.c_int32, [vp, vp, C.POINTER(CLoadStep), C.c_int32, ip]),
        "lpmgpu_batch_add_fatigue": (C.c_int32, [vp, vp, C.POINTER(CLoadStep), C.c_int32, C.POINTER(CLoadStep),
                                                 C.c_int32, C.c_int32, dp, ip]),
        "lpmgpu_batch_round": (C.c_int32, [vp, ip]),
        "lpmgpu_batch_run": (C.c_int32, [vp]),
        "lpmgpu_batch_member": (C.c_int32, [vp, C.c_int32, C.POINTER(MemberInfo)]),
        "lpmgpu_batch_member_steps": (C.c_int32, [vp, C.c_int32, C.POINTER(Stats), C.c_int32, ip]),
        "lpmgpu_batch_remove": (C.c_int32, [vp, C.c_int32]),
        "lpmgpu_batch_get_stats": (C.c_int32, [vp, C.POINTER(BatchStats)]),
        "lpmgpu_batch_set_slice": (C.c_int32, [vp, C.c_int64]),
        "lpmgpu_batch_set_lanes": (C.c_int32, [vp, C.c_int32]),
        "lpmgpu_batch_set_solo_bytes": (C.c_int32, [vp, C.c_int64]),
        "lpmgpu_estimate_bytes": (C.c_int32, [C.POINTER(Desc), lp]),
        "lpmgpu_server_create": (C.c_int32, [C.c_int32, C.c_int64, C.POINTER(vp)]),
        "lpmgpu_server_destroy": (C.c_int32, [vp]),
        "lpmgpu_server_set_slice": (C.c_int32, [vp, C.c_int64]),
        "lpmgpu_server_set_lanes": (C.c_int32, [vp, C.c_int32]),
        "lpmgpu_server_set_solo_bytes": (C.c_int32, [vp, C.c_int64]),
        "lpmgpu_server_submit": (C.c_int32, [vp, C.POINTER(Desc), C.POINTER(CLoadStep), C.c_int32, lp]),
        "lpmgpu_server_submit_fatigue": (C.c_int32, [vp, C.POINTER(Desc), C.POINTER(CLoadStep), C.c_int32,
                                                     C.POINTER(CLoadStep), C.c_int32, C.c_int32, dp, lp]),
        "lpmgpu_server_poll": (C.c_int32, [vp, C.c_int64, C.POINTER(RequestInfo)]),
        "lpmgpu_server_wait": (C.c_int32, [vp, C.c_int64, C.c_double, C.POINTER(RequestInfo)]),
        "lpmgpu_server_result": (C.c_int32, [vp, C.c_int64, dp, C.c_int64]),
        "lpmgpu_server_get_stats": (C.c_int32, [vp, C.POINTER(ServerStats)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def _dp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int32))


def _lp(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_int64))


def _check(status, where):
    if status != OK:
        raise LpmGpuError(status, where)


# ---------------------------------------------------------------------------- unit cell / generators
class UnitCell:
    """include/unit_cell.h:27-122 (constants only; the device computes the same ones)."""

    def __init__(self, lattice: LatticeType, radius: float):
        self.lattice = LatticeType(lattice)
        self.radius = float(radius)
        r, s2, s3 = self.radius, np.sqrt(2.0), np.sqrt(3.0)
        if self.lattice == LatticeType.Square2D:
            self.dim, self.nneighbors, self.neighbor_cutoff = 2, 8, [2.0 * r, 2.0 * s2 * r]
        elif self.lattice == LatticeType.Hexagon2D:
            self.dim, self.nneighbors, self.neighbor_cutoff = 2, 12, [2.0 * r, 2.0 * s3 * r]
        elif self.lattice in (LatticeType.SimpleCubic3D, LatticeType.FCC3D):
            self.dim, self.nneighbors, self.neighbor_cutoff = 3, 18, [2.0 * r, 2.0 * s2 * r]
        else:
            self.dim, self.nneighbors, self.neighbor_cutoff = 3, 14, [2.0 * r, 4.0 / s3 * r]


def createRMatrix(eulerflag: int, angles: Sequence[float]):
    """include/utilities.h:15-91; returned as (flag, angles) for the generators."""
    return (int(eulerflag), np.ascontiguousarray(angles, dtype=np.float64))


def _generate(lattice: LatticeType, box, cell: UnitCell, R) -> np.ndarray:
    L = lib()
    b = np.ascontiguousarray(box, dtype=np.float64)
    flag, ang = R if R is not None else (0, np.zeros(3))
    cnt = C.c_int64(0)
    _check(L.lpmgpu_generate_lattice(int(lattice), cell.radius, _dp(b), flag, _dp(ang), None, 0, C.byref(cnt)),
           "lpmgpu_generate_lattice")
    out = np.zeros((cnt.value, 3))
    _check(L.lpmgpu_generate_lattice(int(lattice), cell.radius, _dp(b), flag, _dp(ang), _dp(out), cnt.value,
                                     C.byref(cnt)), "lpmgpu_generate_lattice")
    return out


def createPlateSQ2D(box, cell, R=None):
    return _generate(LatticeType.Square2D, box, cell, R)


def createPlateHEX2D(box, cell, R=None):
    return _generate(LatticeType.Hexagon2D, box, cell, R)


def createCuboidSC3D(box, cell, R=None):
    return _generate(LatticeType.SimpleCubic3D, box, cell, R)


def createCuboidFCC3D(box, cell, R=None):
    return _generate(LatticeType.FCC3D, box, cell, R)


def createCuboidBCC3D(box, cell, R=None):
    """No counterpart in the reference: corner + body-centre sites, nearest distance 2r."""
    return _generate(LatticeType.BCC3D, box, cell, R)


# ---------------------------------------------------------------------------- assembly and loads
@dataclass
class Material:
    """Arguments of setParticleProperty (particle_elastic.h:70, particle_j2plasticity.h:155,
    particle_elastic_damage.h:176, particle_fatigue_hcf.h:163)."""
    plane_stress: bool = False
    E: float = 69e3
    mu: float = 0.3
    critical_bstrain: float = 1.0
    sigmay: float = 0.0
    xi: float = 0.0
    H: float = 0.0
    A: float = 0.0
    nonlocal_L: float = 0.0
    # ParticleElasticDamage: damage surface k0 + k1 D on the strain energy density, the
    # compression/tension ratio and the damage threshold
    k0: float = 0.0
    k1: float = 1.0
    comp_tensile_ratio: float = 10.0
    damage_threshold: float = 1.0
    # ParticleFatigueHCF (particle_fatigue_hcf.h:163-205): damage rate A pow(max energy, B)
    # pow(energy range, d); the fatigue limit ratio is kept but unused, as in the reference
    fatigue_A: float = 0.0
    fatigue_B: float = 0.0
    fatigue_d: float = 0.0
    fatigue_limit_ratio: float = 1.108
    # setParticleProperty's (C11, C12, C44) overload (particle_elastic.h:110-140): C11 > 0 takes
    # the bond coefficients from these constants instead of E, mu and plane_stress
    C11: float = 0.0
    C12: float = 0.0
    C44: float = 0.0


def _read_dump(path: str):
    """LAMMPS-style dump as Assembly::readDump reads it (include/assembly.h:338-388): three
    header lines, the particle count, one line, three box lines, one line, then
    "id type x y z" records."""
    if not os.path.exists(path):
        raise FileNotFoundError(f"'{path}' does not exist!")
    with open(path) as f:
        lines = f.read().splitlines()
    n = int(lines[3].split()[0])
    box = [float(v) for k in (5, 6, 7) for v in lines[k].split()[:2]]
    rec = np.array([ln.split()[:5] for ln in lines[9:9 + n] if ln.strip()], dtype=np.float64).reshape(-1, 5)
    if len(rec) != n or not np.array_equal(rec[:, 0], np.arange(n)):
        raise ValueError(f"{path}: expected {n} particles with ids 0..{n - 1} in file order")
    return box, rec[:, 1].astype(np.int32), np.ascontiguousarray(rec[:, 2:5])


class Assembly:
    """Particle system built from coordinates (include/assembly.h:98-106).  The bonds and
    connections are built on the device when the solver is constructed."""

    def __init__(self, xyz, box, cell: UnitCell, ptype: ParticleType = ParticleType.Elastic):
        self.xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
        self.box = list(box)
        self.cell = cell
        self.ptype = ParticleType(ptype)
        self.nparticle = len(self.xyz)
        self.type = np.zeros(self.nparticle, dtype=np.int32)
        self.material = Material()
        # optional explicit bonds (Assembly(dumpFile, bondFile) / pre-cracks), per-bond
        # coefficients and initial bond damage, all in (particle, layer-0 then layer-1) order
        self.bonds = None          # (nb0[n], nb1[n], p2[nbonds])
        self.bond_kn = self.bond_tv = self.bond_damage = None
        self.nonlocal_cutoff_ratio = 0.0  # > 0 once searchNonlocalNeighbors ran

    def searchNonlocalNeighbors(self, cutoff_ratio: float):
        """Assembly::searchNonlocalNeighbors (include/assembly.h:118-130): every particle within
        cutoff_ratio x nonlocal_L of a particle is its nonlocal neighbour.  The search runs on the
        device when the solver is constructed."""
        self.nonlocal_cutoff_ratio = float(cutoff_ratio)

    @classmethod
    def fromDump(cls, dumpFile: str, cell: UnitCell, ptype: ParticleType = ParticleType.Elastic,
                 bondFile: str = None) -> "Assembly":
        """Assembly(dumpFile, cell, ptype) and Assembly(dumpFile, bondFile, cell, ptype)
        (include/assembly.h:74-95): ids, types and coordinates from a LAMMPS-style dump
        (readDump, assembly.h:338-388); bonds from the bond file (readBond) or, without one, from
        the device's bond search (createBonds).  Particle ids must run 0..n-1 in file order."""
        box, types, xyz = _read_dump(dumpFile)
        a = cls(xyz, box, cell, ptype)
        a.type = types
        if bondFile is not None:
            a.readBond(bondFile)
        return a

    def readBond(self, bondFile: str):
        """Assembly::readBond (include/assembly.h:391-424): one "id layer p1 p2" line per bond;
        each bond joins p1's list of its layer in file order."""
        if not os.path.exists(bondFile):
            raise FileNotFoundError(f"'{bondFile}' does not exist!")
        rows = np.loadtxt(bondFile, dtype=np.int64, ndmin=2).reshape(-1, 4)
        layer, p1, p2 = rows[:, 1], rows[:, 2], rows[:, 3]
        n = self.nparticle
        if rows.size and (layer.min() < 0 or layer.max() > 1 or p1.min() < 0 or p1.max() >= n
                          or p2.min() < 0 or p2.max() >= n):
            raise ValueError(f"{bondFile}: layer outside 0..1 or particle id outside 0..{n - 1}")
        order = np.lexsort((layer, p1))  # stable: file order inside each (p1, layer) list
        nb0 = np.bincount(p1[layer == 0], minlength=n).astype(np.int32)
        nb1 = np.bincount(p1[layer == 1], minlength=n).astype(np.int32)
        self.bonds = (nb0, nb1, p2[order].astype(np.int32))

    def writeBond(self, bondFile: str):
        """Assembly::writeBond (include/assembly.h:269-283) for explicit bond lists."""
        if self.bonds is None:
            raise ValueError("writeBond needs explicit bond lists (readBond or Assembly.bonds)")
        nb0, nb1, p2 = (np.asarray(a, dtype=np.int64) for a in self.bonds)
        nb = nb0 + nb1
        start = np.concatenate([[0], np.cumsum(nb)[:-1]]).astype(np.int64)
        layer = (np.arange(len(p2)) - np.repeat(start, nb) >= np.repeat(nb0, nb)).astype(np.int64)
        rows = np.stack([np.arange(len(p2)), layer, np.repeat(np.arange(len(nb)), nb), p2], axis=1)
        np.savetxt(bondFile, rows, fmt="%d")

    def setParticleProperty(self, nonlocal_L, is_plane_stress, E, mu, *rest):
        """setParticleProperty of the assembly's particle type.  With a bool second argument, the
        isotropic overloads:
        Elastic: (nonlocal_L, is_plane_stress, E, mu, critical_bstrain) (particle_elastic.h:71);
        J2: (nonlocal_L, is_plane_stress, E, mu, sigmay, xi, H, A, critical_bstrain)
        (particle_j2plasticity.h:155);
        ElasticDamage: (nonlocal_L, is_plane_stress, E, mu, k0, k1, ct_ratio, d_thres)
        (particle_elastic_damage.h:176);
        FatigueHCF: (nonlocal_L, is_plane_stress, E, mu, A, B, d, d_thres, f_lmt_ratio)
        (particle_fatigue_hcf.h:163).
        With a number there, the cubic-constant overloads: Elastic (nonlocal_L, C11, C12, C44,
        critical_bstrain) (particle_elastic.h:111); ElasticDamage (nonlocal_L, C11, C12, C44, k0, k1,
        ct_ratio, d_thres) (particle_elastic_damage.h:219)."""
        if not isinstance(is_plane_stress, (bool, np.bool_)):
            C11, C12, C44 = float(is_plane_stress), float(E), float(mu)
            m = Material(nonlocal_L=float(nonlocal_L), C11=C11, C12=C12, C44=C44)
            if self.ptype == ParticleType.ElasticDamage:
                m.k0, m.k1, m.comp_tensile_ratio, m.damage_threshold = map(float, rest)
            elif self.ptype == ParticleType.Elastic:
                (m.critical_bstrain,) = map(float, rest)
            else:
                raise ValueError("the (C11, C12, C44) overload exists for elastic and elastic-damage particles")
            self.material = m
            return
        m = Material(plane_stress=bool(is_plane_stress), E=float(E), mu=float(mu), nonlocal_L=float(nonlocal_L))
        if self.ptype == ParticleType.J2Plasticity:
            m.sigmay, m.xi, m.H, m.A, m.critical_bstrain = map(float, rest)
        elif self.ptype == ParticleType.ElasticDamage:
            m.k0, m.k1, m.comp_tensile_ratio, m.damage_threshold = map(float, rest)
        elif self.ptype == ParticleType.FatigueHCF:
            m.fatigue_A, m.fatigue_B, m.fatigue_d, m.damage_threshold, m.fatigue_limit_ratio = map(float, rest)
        else:
            (m.critical_bstrain,) = map(float, rest)
        self.material = m

    def group(self, mask) -> np.ndarray:
        return np.nonzero(np.asarray(mask))[0].astype(np.int32)


_FLAG = {"x": 0, "y": 1, "z": 2}


@dataclass
class DispBC:
    group: np.ndarray
    load_mode: LoadMode
    flag: str
    step: float

    def cutHalf(self):
        self.step /= 2.0


@dataclass
class ForceBC:
    group: np.ndarray
    load_mode: LoadMode
    fx: float
    fy: float
    fz: float

    def cutHalf(self):
        self.fx /= 2.0
        self.fy /= 2.0
        self.fz /= 2.0


@dataclass
class LoadStep:
    dispBCs: List[DispBC] = field(default_factory=list)
    forceBCs: List[ForceBC] = field(default_factory=list)

    def loadCutHalf(self):
        for d in self.dispBCs:
            d.cutHalf()
        for f in self.forceBCs:
            f.cutHalf()


# ---------------------------------------------------------------------------- fatigue loading
class FatigueLoadType(enum.IntEnum):
    """include/load_step_fatigue.h:14-20"""
    LoadUniaxialDisp = 0
    LoadUniaxialForce = 1
    LoadDogBoneDisp = 2
    LoadCTForce = 3


class TimeMapMode(enum.IntEnum):
    """include/lpm.h:85-89"""
    Linear = 0
    Exponential = 1


def LoadUniaxialForce(fy, left_group, top_group, bottom_group) -> LoadStep:
    """include/load_step_fatigue.h:23-36"""
    return LoadStep([DispBC(left_group, LoadMode.Relative, "x", 0.0), DispBC(bottom_group, LoadMode.Relative, "y", 0.0)],
                    [ForceBC(top_group, LoadMode.Relative, 0.0, fy, 0.0)])


def LoadUniaxialDisp(dy, left_group, top_group, bottom_group) -> LoadStep:
    """include/load_step_fatigue.h:38-51"""
    return LoadStep([DispBC(left_group, LoadMode.Relative, "x", 0.0), DispBC(top_group, LoadMode.Relative, "y", dy),
                     DispBC(bottom_group, LoadMode.Relative, "y", 0.0)], [])


def LoadDogBoneDisp(x, y, z, group1, group2) -> LoadStep:
    """include/load_step_fatigue.h:53-69"""
    return LoadStep([DispBC(group1, LoadMode.Relative, "x", x), DispBC(group1, LoadMode.Relative, "y", y),
                     DispBC(group1, LoadMode.Relative, "z", z), DispBC(group2, LoadMode.Relative, "x", 0.0),
                     DispBC(group2, LoadMode.Relative, "y", 0.0), DispBC(group2, LoadMode.Relative, "z", 0.0)], [])


def LoadCTForce(fy, mid_group, top_group, bottom_group) -> LoadStep:
    """include/load_step_fatigue.h:71-87"""
    return LoadStep([DispBC(mid_group, LoadMode.Relative, "y", 0.0), DispBC(top_group, LoadMode.Relative, "x", 0.0),
                     DispBC(bottom_group, LoadMode.Relative, "x", 0.0)],
                    [ForceBC(top_group, LoadMode.Relative, 0.0, fy, 0.0),
                     ForceBC(bottom_group, LoadMode.Relative, 0.0, -fy, 0.0)])


def func_dNdt_linear(tau: float) -> int:
    """include/solver_fatigue.h:60-63: (int)(1 / tau)"""
    return int(1 / tau)


def func_dNdt_exponental(tau: float, t: float) -> int:
    """include/solver_fatigue.h:65-68: (int)(1 / tau * exp(t / tau))"""
    return int(1 / tau * math.exp(t / tau))


def generateLoadCycle(ltype: FatigueLoadType, load_spectrum: Sequence[float], N: int, n_interval: int,
                      pt_groups: Sequence[np.ndarray]) -> List[LoadStep]:
    """SolverFatigue::generateLoadCycle (include/solver_fatigue.h:128-180): the cycle from
    spectrum values f0 = [2N], f1 = [2N+1], f2 = [2N+2] as n_interval steps of (f1 - f0) / n_interval
    then n_interval steps of (f2 - f1) / n_interval."""
    f0, f1, f2 = (float(load_spectrum[2 * N + k]) for k in range(3))
    g = list(pt_groups)
    make = {FatigueLoadType.LoadUniaxialDisp: lambda v: LoadUniaxialDisp(v, g[0], g[1], g[2]),
            FatigueLoadType.LoadUniaxialForce: lambda v: LoadUniaxialForce(v, g[0], g[1], g[2]),
            FatigueLoadType.LoadDogBoneDisp: lambda v: LoadDogBoneDisp(0, v, 0, g[0], g[1]),
            FatigueLoadType.LoadCTForce: lambda v: LoadCTForce(v, g[0], g[1], g[2])}[FatigueLoadType(ltype)]
    return ([make((f1 - f0) / n_interval) for _ in range(n_interval)] +
            [make((f2 - f1) / n_interval) for _ in range(n_interval)])


class _CStep:
    """Keeps the ctypes arrays of one load step alive for a call."""

    def __init__(self, step: LoadStep):
        for bc in list(step.dispBCs) + list(step.forceBCs):
            if bc.load_mode != LoadMode.Relative:
                raise ValueError("only LoadMode.Relative is supported (Absolute teleports particles in the "
                                 "reference, solver.h:140-141)")
        self.keep = []
        nd, nf = len(step.dispBCs), len(step.forceBCs)
        self.d = (CDispBC * max(nd, 1))()
        self.f = (CForceBC * max(nf, 1))()
        for q, bc in enumerate(step.dispBCs):
            ids = np.ascontiguousarray(bc.group, dtype=np.int32)
            self.keep.append(ids)
            self.d[q] = CDispBC(_ip(ids), len(ids), _FLAG[bc.flag] if isinstance(bc.flag, str) else int(bc.flag),
                                float(bc.step))
        for q, bc in enumerate(step.forceBCs):
            ids = np.ascontiguousarray(bc.group, dtype=np.int32)
            self.keep.append(ids)
            self.f[q] = CForceBC(_ip(ids), len(ids), float(bc.fx), float(bc.fy), float(bc.fz))
        self.s = CLoadStep(self.d, nd, self.f, nf)


# ---------------------------------------------------------------------------- solver
def _pack_desc(ass: Assembly, undamaged_pt_type=-1, max_iter=30, tol_iter=1e-5, precision=0, cg_rtol=1e-12,
               cg_atol=1e-12, cg_maxit=0, device=0, tangent=False, direct=0):
    """lpmgpu_desc of an Assembly and solver settings; returns (desc, arrays the desc points into)."""
    m = ass.material
    d = Desc()
    keep = [np.ascontiguousarray(ass.xyz, dtype=np.float64), np.ascontiguousarray(ass.type, dtype=np.int32)]
    d.lattice, d.ptype, d.n = int(ass.cell.lattice), int(ass.ptype), ass.nparticle
    d.xyz, d.type = _dp(keep[0]), _ip(keep[1])
    d.radius, d.plane_stress = ass.cell.radius, int(m.plane_stress)
    d.E, d.mu, d.critical_bstrain = m.E, m.mu, m.critical_bstrain
    d.sigmay, d.xi, d.H, d.A, d.nonlocal_L = m.sigmay, m.xi, m.H, m.A, m.nonlocal_L
    d.undamaged_type, d.max_iter, d.tol_iter = int(undamaged_pt_type), int(max_iter), float(tol_iter)
    d.cg_rtol, d.cg_atol, d.cg_maxit = float(cg_rtol), float(cg_atol), int(cg_maxit)
    d.precision, d.device = int(precision), int(device)
    d.tangent = int(bool(tangent))
    d.direct = int(direct)
    d.nonlocal_cutoff_ratio = float(getattr(ass, "nonlocal_cutoff_ratio", 0.0))
    d.k0, d.k1, d.comp_tensile_ratio, d.damage_threshold = m.k0, m.k1, m.comp_tensile_ratio, m.damage_threshold
    d.fatigue_A, d.fatigue_B, d.fatigue_d = m.fatigue_A, m.fatigue_B, m.fatigue_d
    d.fatigue_limit_ratio = m.fatigue_limit_ratio
    d.C11, d.C12, d.C44 = m.C11, m.C12, m.C44
    if ass.bonds is not None:
        nb0, nb1, p2 = (np.ascontiguousarray(a, dtype=np.int32) for a in ass.bonds)
        keep += [nb0, nb1, p2]
        d.bond_nb0, d.bond_nb1, d.bond_p2 = _ip(nb0), _ip(nb1), _ip(p2)
    for name in ("bond_kn", "bond_tv", "bond_damage"):
        arr = getattr(ass, name)
        if arr is not None:
            a = np.ascontiguousarray(arr, dtype=np.float64)
            keep.append(a)
            setattr(d, name, _dp(a))
    return d, keep


class GpuProblem:
    """One device-resident problem: the handle of include/lpmgpu.h."""

    def __init__(self, ass: Assembly, undamaged_pt_type=-1, max_iter=30, tol_iter=1e-5,
                 precision: Precision = Precision.FP64, cg_rtol=1e-12, cg_atol=1e-12, cg_maxit=0, device=0,
                 tangent: bool = False, direct: int = 0):
        """tangent: re-assemble K from the current state before every Newton solve (the
        default keeps K fixed per load step, as SolverStatic does).  direct: the linear solver
        of the Newton iterations, 0 the CG, 1 the band Cholesky, 2 the band Cholesky when its
        band fits, else the CG (lpmgpu_desc.direct)."""
        L = lib()
        self.ass = ass
        d, self._keep = _pack_desc(ass, undamaged_pt_type, max_iter, tol_iter, precision, cg_rtol, cg_atol, cg_maxit,
                                   device, tangent, direct)
        h = C.c_void_p()
        _check(L.lpmgpu_create(C.byref(d), C.byref(h)), "lpmgpu_create")
        self._h = h
        s = Sizes()
        _check(L.lpmgpu_get_sizes(h, C.byref(s)), "lpmgpu_get_sizes")
        self.sizes = {k: getattr(s, k) for k, _ in s._fields_}
        self.n, self.dim = s.n, s.dim
        self.nsv = {ParticleType.J2Plasticity: 7, ParticleType.FatigueHCF: 3}.get(ass.ptype, 1)

    def close(self):
        if getattr(self, "_h", None):
            lib().lpmgpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- topology and matrices
    def topology(self):
        n, nb, nnzb = self.n, self.sizes["nbonds"], self.sizes["nnzb"]
        nb0, nb1, p2 = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(nb, np.int32)
        nconn, nlq, conns = np.zeros(n, np.int32), np.zeros(n, np.int32), np.zeros(nnzb, np.int32)
        _check(lib().lpmgpu_get_topology(self._h, _ip(nb0), _ip(nb1), _ip(p2), _ip(nconn), _ip(nlq), _ip(conns)),
               "lpmgpu_get_topology")
        return {"nb0": nb0, "nb1": nb1, "bond_p2": p2, "nconn": nconn, "nlq": nlq, "conns": conns}

    def export_csr(self):
        nnz = self.sizes["nnz_upper"]
        Kp = np.zeros(self.n + 1, np.int64)
        IK = np.zeros(self.dim * self.n + 1, np.int64)
        JK = np.zeros(nnz, np.int64)
        K = np.zeros(nnz)
        _check(lib().lpmgpu_export_ref_csr(self._h, _lp(Kp), _lp(IK), _lp(JK), _dp(K)), "lpmgpu_export_ref_csr")
        return Kp, IK, JK, K

    # ---- physics steps
    def update_force_state(self):
        _check(lib().lpmgpu_update_force_state(self._h), "lpmgpu_update_force_state")

    def update_state_var(self):
        _check(lib().lpmgpu_update_state_var(self._h), "lpmgpu_update_state_var")

    def update_rr(self) -> float:
        v = C.c_double(0)
        _check(lib().lpmgpu_update_rr(self._h, C.byref(v)), "lpmgpu_update_rr")
        return v.value

    def assemble(self, apply_bc=True):
        _check(lib().lpmgpu_assemble(self._h, int(apply_bc)), "lpmgpu_assemble")

    def nonlocal_lists(self):
        """(count per particle, concatenated ids) of the nonlocal neighbour lists, or None when the
        problem has none (lpmgpu_get_nonlocal)."""
        total = C.c_int64(0)
        _check(lib().lpmgpu_get_nonlocal(self._h, None, None, C.byref(total)), "lpmgpu_get_nonlocal")
        if total.value == 0:
            return None
        cnt = np.zeros(self.n, np.int32)
        ids = np.zeros(total.value, np.int32)
        _check(lib().lpmgpu_get_nonlocal(self._h, _ip(cnt), _ip(ids), C.byref(total)), "lpmgpu_get_nonlocal")
        return cnt, ids

    def solve_direct(self):
        """The band Cholesky solve of the current K and residual (lpmgpu_solve_direct): the
        displacement increment."""
        disp = np.zeros(self.dim * self.n)
        st = Stats()
        _check(lib().lpmgpu_solve_direct(self._h, _dp(disp), C.byref(st)), "lpmgpu_solve_direct")
        return disp, st.as_dict()

    def solve_linear(self):
        disp = np.zeros(self.dim * self.n)
        st = Stats()
        _check(lib().lpmgpu_solve_linear(self._h, _dp(disp), C.byref(st)), "lpmgpu_solve_linear")
        return disp, st.as_dict()

    def apply_load_step(self, step: LoadStep):
        cs = _CStep(step)
        _check(lib().lpmgpu_apply_load_step(self._h, C.byref(cs.s)), "lpmgpu_apply_load_step")

    def solve_problem_step(self, step: LoadStep):
        cs = _CStep(step)
        st = Stats()
        r = lib().lpmgpu_solve_problem_step(self._h, C.byref(cs.s), C.byref(st))
        if r not in (OK, ERR_NEWTON):
            _check(r, "lpmgpu_solve_problem_step")
        return r == OK, st.as_dict()

    def solve_load_step(self, step: LoadStep):
        cs = _CStep(step)
        st = Stats()
        r = lib().lpmgpu_solve_load_step(self._h, C.byref(cs.s), C.byref(st))
        if r not in (OK, ERR_CUTS):
            _check(r, "lpmgpu_solve_load_step")
        return r == OK, st.as_dict()

    # ---- SolverFatigue steps (include/solver_fatigue.h)
    def fatigue_solve_step(self, step: LoadStep):
        """SolverFatigue::solveProblemStep: (converged, stats)."""
        cs = _CStep(step)
        st = Stats()
        r = lib().lpmgpu_fatigue_solve_step(self._h, C.byref(cs.s), C.byref(st))
        if r not in (OK, ERR_NEWTON):
            _check(r, "lpmgpu_fatigue_solve_step")
        return r == OK, st.as_dict()

    def fatigue_static_step(self, step: LoadStep):
        """One load step of SolverFatigue::solveProblemStatic: (converged, stats)."""
        cs = _CStep(step)
        st = Stats()
        r = lib().lpmgpu_fatigue_static_step(self._h, C.byref(cs.s), C.byref(st))
        if r not in (OK, ERR_CUTS):
            _check(r, "lpmgpu_fatigue_static_step")
        return r == OK, st.as_dict()

    def fatigue_update_damage(self, dNdt: float) -> bool:
        """SolverFatigue::updateFatigueDamage: True when some damage moved by more than 1e-3."""
        flag = C.c_int32(0)
        _check(lib().lpmgpu_fatigue_update_damage(self._h, float(dNdt), C.byref(flag)), "lpmgpu_fatigue_update_damage")
        return bool(flag.value)

    def fatigue_cycle(self, steps: Sequence[LoadStep], dNdt: float):
        """SolverFatigue::solveProblemOneCycle: (any_damaged, stats); stats["cuts"] counts the
        steps whose Newton iteration did not converge (the reference carries on from them)."""
        cs = [_CStep(x) for x in steps]
        arr = (CLoadStep * max(len(cs), 1))(*[c.s for c in cs])
        st = Stats()
        flag = C.c_int32(0)
        _check(lib().lpmgpu_fatigue_cycle(self._h, arr, len(cs), float(dNdt), C.byref(st), C.byref(flag)),
               "lpmgpu_fatigue_cycle")
        return bool(flag.value), st.as_dict()

    def autotune(self, iterations: int = 50) -> dict:
        """Times the CG kernel on this problem for several grid sizes and keeps the fastest
        (lpmgpu_autotune).  Call between load steps: it re-assembles K from the current state."""
        r = TuneResult()
        _check(lib().lpmgpu_autotune(self._h, int(iterations), C.byref(r)), "lpmgpu_autotune")
        return r.as_dict()

    def set_cg_grid(self, grid: int):
        """Blocks per CG launch; 0 restores the default (one block per SM, at most one per slice)."""
        _check(lib().lpmgpu_set_cg_grid(self._h, int(grid)), "lpmgpu_set_cg_grid")

    def set_assembly_exact(self, exact: bool = True):
        """The bit-exact stiffness kernel (reference operator order) instead of the default fast
        form (within rounding of the reference; lpmgpu_set_assembly_exact)."""
        _check(lib().lpmgpu_set_assembly_exact(self._h, int(bool(exact))), "lpmgpu_set_assembly_exact")

    def set_wait_limit_ns(self, ns: int):
        """Time limit of each grid-barrier wait in this problem's CG kernel; 0 restores the
        default of 4 s (lpmgpu_set_wait_limit_ns).  A solve whose wait exceeds it raises
        LpmGpuError with LPMGPU_ERR_TIMEOUT, and the problem stays usable."""
        _check(lib().lpmgpu_set_wait_limit_ns(self._h, int(ns)), "lpmgpu_set_wait_limit_ns")

    def store_state(self):
        _check(lib().lpmgpu_store_state(self._h), "lpmgpu_store_state")

    def reset_state(self):
        _check(lib().lpmgpu_reset_state(self._h), "lpmgpu_reset_state")

    def set_xyz(self, xyz):
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        _check(lib().lpmgpu_set_xyz(self._h, _dp(a)), "lpmgpu_set_xyz")

    def state(self, fields=("xyz", "pin", "stress", "damage", "damage_visual", "state_var", "bdamage")):
        n = self.n
        shapes = {"xyz": (n, 3), "pin": (n, 3), "stress": (n, 6), "damage": (n,), "damage_visual": (n,),
                  "state_var": (n, self.nsv), "bdamage": (self.sizes["nbonds"],)}
        out = {k: np.zeros(shapes[k]) for k in fields}
        args = [_dp(out.get(k)) for k in ("xyz", "pin", "stress", "damage", "damage_visual", "state_var",
                                          "bdamage")]
        _check(lib().lpmgpu_read_state(self._h, *args), "lpmgpu_read_state")
        return out

    def residual(self):
        r = np.zeros(self.dim * self.n)
        _check(lib().lpmgpu_read_residual(self._h, _dp(r)), "lpmgpu_read_residual")
        return r

    def counters(self):
        c = Counters()
        _check(lib().lpmgpu_get_counters(self._h, C.byref(c)), "lpmgpu_get_counters")
        return c.as_dict()

    def dump_write(self, path: str, step: int, box, threads: int = 0, async_: bool = True):
        """lpmgpu_dump_write: appends the current state as one step of the reference's dump text
        (Assembly::writeDump, include/assembly.h:310-335); async_ overlaps the formatting with the
        caller's next device work (lpmgpu_dump_flush waits for it)."""
        b = np.ascontiguousarray(box, dtype=np.float64)
        _check(lib().lpmgpu_dump_write(self._h, os.fsencode(path), int(step), _dp(b), int(threads), int(bool(async_))),
               "lpmgpu_dump_write")

    def dump_flush(self):
        _check(lib().lpmgpu_dump_flush(self._h), "lpmgpu_dump_flush")

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        _check(lib().lpmgpu_get_stream(self._h, C.byref(s)), "lpmgpu_get_stream")
        return s.value or 0

    def read_xyz_into(self, out: np.ndarray):
        """Device-to-host copy of the positions into a caller buffer (n x 3, float64)."""
        _check(lib().lpmgpu_read_state(self._h, _dp(out), None, None, None, None, None, None), "lpmgpu_read_state")

    def phase_times(self):
        t = np.zeros(4)
        _check(lib().lpmgpu_get_phase_times(self._h, _dp(t)), "lpmgpu_get_phase_times")
        return {"force_s": t[0], "assembly_s": t[1], "linear_s": t[2], "other_s": t[3]}


def format_dump(path: str, step: int, box, xyz, xyz_initial, stress, damage, damage_visual, state_var,
                type=None, threads: int = 0):
    """lpmgpu_format_dump: one step of the reference's dump text (Assembly::writeDump,
    include/assembly.h:310-335) for host arrays, appended to path.  Needs no device."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1, 3)
    n = len(xyz)
    sv = np.ascontiguousarray(state_var, dtype=np.float64).reshape(n, -1)
    t = None if type is None else np.ascontiguousarray(type, dtype=np.int32)
    arr = [np.ascontiguousarray(a, dtype=np.float64) for a in (box, xyz_initial, stress, damage, damage_visual)]
    _check(lib().lpmgpu_format_dump(os.fsencode(path), int(step), n, _ip(t), _dp(arr[0]), _dp(xyz), _dp(arr[1]),
                                    _dp(arr[2]), _dp(arr[3]), _dp(arr[4]), _dp(sv), sv.shape[1], int(threads)),
           "lpmgpu_format_dump")


class Batch:
    """Many problems advanced together (lpmgpu_batch_*): each member runs its whole load path
    as repeated GpuProblem.solve_load_step calls would, and all members' Newton systems of a
    round go through one persistent CG launch."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().lpmgpu_batch_create(int(device), C.byref(h)), "lpmgpu_batch_create")
        self._h = h
        self._problems = {}

    def add(self, problem: "GpuProblem", steps: Sequence[LoadStep]) -> int:
        cs = [_CStep(s) for s in steps]
        arr = (CLoadStep * max(len(cs), 1))(*[c.s for c in cs])
        mid = C.c_int32(-1)
        _check(lib().lpmgpu_batch_add(self._h, problem._h, arr, len(cs), C.byref(mid)), "lpmgpu_batch_add")
        self._problems[mid.value] = problem
        return mid.value

    def add_fatigue(self, problem: "GpuProblem", static_steps: Sequence[LoadStep],
                    cycles: Sequence[Sequence[LoadStep]], dndt: Sequence[float]) -> int:
        """A fatigue member (lpmgpu_batch_add_fatigue): the static steps as
        SolverFatigue::solveProblemStatic runs them, then each cycle (equal lengths) as
        solveProblemOneCycle with its dN/dt."""
        if len(cycles) != len(dndt) or len({len(c) for c in cycles}) > 1:
            raise ValueError("one dN/dt per cycle, and cycles of equal length")
        cs = [_CStep(s) for s in static_steps]
        cc = [_CStep(s) for cyc in cycles for s in cyc]
        a_s = (CLoadStep * max(len(cs), 1))(*[c.s for c in cs])
        a_c = (CLoadStep * max(len(cc), 1))(*[c.s for c in cc])
        d = np.ascontiguousarray(dndt, dtype=np.float64) if len(dndt) else np.zeros(1)
        mid = C.c_int32(-1)
        _check(lib().lpmgpu_batch_add_fatigue(self._h, problem._h, a_s, len(cs), a_c, len(cycles[0]) if cycles else 0,
                                              len(cycles), _dp(d), C.byref(mid)), "lpmgpu_batch_add_fatigue")
        self._problems[mid.value] = problem
        return mid.value

    def set_slice(self, iterations: int):
        """CG iterations per batched launch before unfinished solves pause (0: no limit)."""
        _check(lib().lpmgpu_batch_set_slice(self._h, int(iterations)), "lpmgpu_batch_set_slice")

    def set_lanes(self, lanes: int):
        """Independent groups of members, each with its own CG launches on a share of the SMs
        (lpmgpu_batch_set_lanes); only while no member is running."""
        _check(lib().lpmgpu_batch_set_lanes(self._h, int(lanes)), "lpmgpu_batch_set_lanes")

    def set_solo_bytes(self, nbytes: int):
        """Members added afterwards whose CG streams at least `nbytes` of matrix per iteration
        solve their linear systems alone through the single-problem CG, between the batched
        launches (lpmgpu_batch_set_solo_bytes); 0 = none."""
        _check(lib().lpmgpu_batch_set_solo_bytes(self._h, int(nbytes)), "lpmgpu_batch_set_solo_bytes")

    def round(self) -> int:
        running = C.c_int32(0)
        _check(lib().lpmgpu_batch_round(self._h, C.byref(running)), "lpmgpu_batch_round")
        return running.value

    def run(self):
        _check(lib().lpmgpu_batch_run(self._h), "lpmgpu_batch_run")

    def member(self, mid: int) -> dict:
        info = MemberInfo()
        _check(lib().lpmgpu_batch_member(self._h, int(mid), C.byref(info)), "lpmgpu_batch_member")
        d = {k: getattr(info, k) for k, _ in MemberInfo._fields_ if k != "total"}
        d["total"] = info.total.as_dict()
        return d

    def member_steps(self, mid: int) -> list:
        cnt = C.c_int32(0)
        _check(lib().lpmgpu_batch_member_steps(self._h, int(mid), None, 0, C.byref(cnt)), "lpmgpu_batch_member_steps")
        arr = (Stats * max(cnt.value, 1))()
        _check(lib().lpmgpu_batch_member_steps(self._h, int(mid), arr, cnt.value, C.byref(cnt)),
               "lpmgpu_batch_member_steps")
        return [arr[k].as_dict() for k in range(cnt.value)]

    def remove(self, mid: int):
        _check(lib().lpmgpu_batch_remove(self._h, int(mid)), "lpmgpu_batch_remove")
        self._problems.pop(mid, None)

    def stats(self) -> dict:
        st = BatchStats()
        _check(lib().lpmgpu_batch_get_stats(self._h, C.byref(st)), "lpmgpu_batch_get_stats")
        return st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib().lpmgpu_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Serving loop (lpmgpu_server_*): submit LPM solves while others run; each is admitted when
    its device memory fits the HBM budget and joins the running batch (continuous batching)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 150 * 10**9):
        h = C.c_void_p()
        _check(lib().lpmgpu_server_create(int(device), int(hbm_budget_bytes), C.byref(h)), "lpmgpu_server_create")
        self._h = h
        self.device = int(device)
        self._n = {}

    @staticmethod
    def estimate_bytes(ass: Assembly, precision: Precision = Precision.FP64) -> int:
        """Device memory the admission test expects the problem to take (lpmgpu_estimate_bytes)."""
        d, keep = _pack_desc(ass, precision=precision)
        out = C.c_int64(0)
        _check(lib().lpmgpu_estimate_bytes(C.byref(d), C.byref(out)), "lpmgpu_estimate_bytes")
        return out.value

    def set_slice(self, iterations: int):
        _check(lib().lpmgpu_server_set_slice(self._h, int(iterations)), "lpmgpu_server_set_slice")

    def set_lanes(self, lanes: int):
        """lpmgpu_server_set_lanes: the batch's lanes, applied once no request is running."""
        _check(lib().lpmgpu_server_set_lanes(self._h, int(lanes)), "lpmgpu_server_set_lanes")

    def set_solo_bytes(self, nbytes: int):
        """lpmgpu_server_set_solo_bytes: the batch's solo threshold for requests joining afterwards."""
        _check(lib().lpmgpu_server_set_solo_bytes(self._h, int(nbytes)), "lpmgpu_server_set_solo_bytes")

    def submit(self, ass: Assembly, steps: Sequence[LoadStep], undamaged_pt_type=-1, max_iter=30, tol_iter=1e-5,
               precision: Precision = Precision.FP64, cg_rtol=1e-12, cg_atol=1e-12, cg_maxit=0,
               tangent: bool = False) -> int:
        d, keep = _pack_desc(ass, undamaged_pt_type, max_iter, tol_iter, precision, cg_rtol, cg_atol, cg_maxit,
                             self.device, tangent)
        cs = [_CStep(s) for s in steps]
        arr = (CLoadStep * max(len(cs), 1))(*[c.s for c in cs])
        rid = C.c_int64(0)
        _check(lib().lpmgpu_server_submit(self._h, C.byref(d), arr, len(cs), C.byref(rid)), "lpmgpu_server_submit")
        self._n[rid.value] = ass.nparticle
        return rid.value

    def submit_fatigue(self, ass: Assembly, static_steps: Sequence[LoadStep], cycles: Sequence[Sequence[LoadStep]],
                       dndt: Sequence[float], undamaged_pt_type=-1, max_iter=30, tol_iter=1e-5,
                       precision: Precision = Precision.FP64, cg_rtol=1e-12, cg_atol=1e-12, cg_maxit=0) -> int:
        """A SolverFatigue run as a request (lpmgpu_server_submit_fatigue): the static steps, then
        the cycles (equal lengths) with their dN/dt."""
        if len(cycles) != len(dndt) or len({len(c) for c in cycles}) > 1:
            raise ValueError("one dN/dt per cycle, and cycles of equal length")
        d, keep = _pack_desc(ass, undamaged_pt_type, max_iter, tol_iter, precision, cg_rtol, cg_atol, cg_maxit,
                             self.device, False)
        cs = [_CStep(s) for s in static_steps]
        cc = [_CStep(s) for cyc in cycles for s in cyc]
        a_s = (CLoadStep * max(len(cs), 1))(*[c.s for c in cs])
        a_c = (CLoadStep * max(len(cc), 1))(*[c.s for c in cc])
        dd = np.ascontiguousarray(dndt, dtype=np.float64) if len(dndt) else np.zeros(1)
        rid = C.c_int64(0)
        _check(lib().lpmgpu_server_submit_fatigue(self._h, C.byref(d), a_s, len(cs), a_c,
                                                  len(cycles[0]) if cycles else 0, len(cycles), _dp(dd),
                                                  C.byref(rid)), "lpmgpu_server_submit_fatigue")
        self._n[rid.value] = ass.nparticle
        return rid.value

    def poll(self, rid: int) -> dict:
        info = RequestInfo()
        _check(lib().lpmgpu_server_poll(self._h, int(rid), C.byref(info)), "lpmgpu_server_poll")
        return info.as_dict()

    def wait(self, rid: int, timeout: float = 600.0) -> dict:
        info = RequestInfo()
        r = lib().lpmgpu_server_wait(self._h, int(rid), float(timeout), C.byref(info))
        if r not in (OK, ERR_NOT_READY):
            _check(r, "lpmgpu_server_wait")
        return info.as_dict()

    def result(self, rid: int) -> np.ndarray:
        out = np.zeros((self._n[rid], 3))
        _check(lib().lpmgpu_server_result(self._h, int(rid), _dp(out), out.size), "lpmgpu_server_result")
        self._n.pop(rid, None)
        return out

    def stats(self) -> dict:
        st = ServerStats()
        _check(lib().lpmgpu_server_get_stats(self._h, C.byref(st)), "lpmgpu_server_get_stats")
        return st.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib().lpmgpu_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class _StiffnessView:
    """``solv.stiffness.K_global / K_pointer / IK / JK`` (stiffness.h:24-26), read on demand."""

    def __init__(self, prob: GpuProblem):
        self._p = prob

    def _load(self):
        self.K_pointer, self.IK, self.JK, self.K_global = self._p.export_csr()

    def __getattr__(self, name):
        if name in ("K_pointer", "IK", "JK", "K_global"):
            self._load()
            return self.__dict__[name]
        raise AttributeError(name)


def _direct_mode(sol_mode) -> int:
    """SolverMode.PARDISO (the reference's direct solve, solver.h:191-274): the CG to a relative
    residual of 1e-12, and the band Cholesky for a system the CG cannot solve (lpmgpu_desc.direct
    = 2); SolverMode.CG: the CG."""
    return 2 if SolverMode(sol_mode) == SolverMode.PARDISO else 0


def _cg_tolerances(sol_mode, rtol, atol):
    """The device CG's squared-norm test for a solver mode: the reference CG's 1e-12 / 1e-12
    (solver.h:312-313), or for PARDISO (a direct solve, solver.h:191-274) 1e-24 relative."""
    pardiso = SolverMode(sol_mode) == SolverMode.PARDISO
    return (rtol if rtol is not None else (1e-24 if pardiso else 1e-12),
            atol if atol is not None else (0.0 if pardiso else 1e-12))


class SolverStatic:
    """SolverStatic<nlayer> (include/solver_static.h:17-29) on the GPU: same constructor
    arguments, same solveProblem(load, start_index) contract; extra keyword arguments choose
    the precision and CG tolerances.  SolverMode.PARDISO, the reference's direct solve, runs the
    device CG to a relative residual of 1e-12 (unless tolerances are given) and the band Cholesky
    for a system the CG cannot solve."""

    def __init__(self, undamaged_pt_type: int, ass: Assembly, stiff_mode=StiffnessMode.Analytical,
                 sol_mode=SolverMode.CG, dumpFile: str = "", max_iter: int = 30, tol: float = 1e-5, *,
                 precision: Precision = Precision.FP64, cg_rtol=None, cg_atol=None, cg_maxit=0, device=0):
        if StiffnessMode(stiff_mode) != StiffnessMode.Analytical:
            raise ValueError("only StiffnessMode.Analytical is on the device path")
        cg_rtol, cg_atol = _cg_tolerances(sol_mode, cg_rtol, cg_atol)
        self.ass = ass
        self.dumpFile = dumpFile
        self.max_NR_iter, self.tol_NR_iter = max_iter, tol
        self.problem = GpuProblem(ass, undamaged_pt_type, max_iter, tol, precision, cg_rtol, cg_atol, cg_maxit,
                                  device, direct=_direct_mode(sol_mode))
        self.stiffness = _StiffnessView(self.problem)
        self.history: List[dict] = []

    def solveProblemStep(self, load_step: LoadStep, dt: float = 1.0) -> bool:
        ok, st = self.problem.solve_problem_step(load_step)
        self.history.append(st)
        return ok

    def solveProblem(self, load: List[LoadStep], start_index: int = 0) -> int:
        """Runs every load step with the reference's halve-and-retry (solver_static.h:65-96).
        Returns the new start_index (the reference updates its int& argument)."""
        for i, step in enumerate(load):
            ok, st = self.problem.solve_load_step(step)
            st["step"] = i + start_index
            self.history.append(st)
            if not ok:
                raise LpmGpuError(ERR_CUTS, f"load step {i + start_index}")
            if self.dumpFile:
                self.writeDump(self.dumpFile, i + start_index)
        self.problem.dump_flush()
        return start_index + len(load)

    def writeDump(self, path: str, step: int):
        """Assembly::writeDump (include/assembly.h:310-335): the native writer, queued behind the
        step's device work (solveProblem flushes before it returns)."""
        self.problem.dump_write(path, step, self.ass.box, async_=True)


class SolverFatigue:
    """SolverFatigue<nlayer> (include/solver_fatigue.h:19-38) on the GPU: the same constructor
    arguments and methods.  Each cycle's steps, the energy updates and the fatigue damage run on
    the device; the cycle loop, the load spectrum and the dN/dt time map are host logic, as in
    the reference."""

    def __init__(self, undamaged_pt_type: int, ass: Assembly, stiff_mode=StiffnessMode.Analytical,
                 sol_mode=SolverMode.CG, t_mode: TimeMapMode = TimeMapMode.Linear, tau: float = 1.0,
                 dumpFile: str = "", max_iter: int = 30, tol: float = 1e-5, *,
                 precision: Precision = Precision.FP64, cg_rtol=None, cg_atol=None, cg_maxit=0, device=0):
        if StiffnessMode(stiff_mode) != StiffnessMode.Analytical:
            raise ValueError("only StiffnessMode.Analytical is on the device path")
        cg_rtol, cg_atol = _cg_tolerances(sol_mode, cg_rtol, cg_atol)
        self.undamaged_pt_type = undamaged_pt_type
        self.ass = ass
        self.t_mode, self.tau = TimeMapMode(t_mode), float(tau)
        self.dumpFile = dumpFile
        self.load_spectrum: List[float] = []
        self.problem = GpuProblem(ass, undamaged_pt_type, max_iter, tol, precision, cg_rtol, cg_atol, cg_maxit,
                                  device, direct=_direct_mode(sol_mode))
        self.stiffness = _StiffnessView(self.problem)
        self.history: List[dict] = []

    def readLoad(self, loadFile: str):
        """SolverFatigue::readLoad (solver_fatigue.h:40-57): every number in the file, in order
        (f_min, then f_max, f_min, ... pairs)."""
        if not os.path.exists(loadFile):
            raise FileNotFoundError(f"'{loadFile}' does not exist!")
        with open(loadFile) as f:
            self.load_spectrum += [float(v) for v in f.read().split()]

    def generateLoadCycle(self, ltype: FatigueLoadType, N: int, n_interval: int, pt_groups) -> List[LoadStep]:
        return generateLoadCycle(ltype, self.load_spectrum, N, n_interval, pt_groups)

    def updateFatigueDamage(self, dNdt: float) -> bool:
        return self.problem.fatigue_update_damage(dNdt)

    def solveProblemStep(self, load_step: LoadStep) -> bool:
        ok, st = self.problem.fatigue_solve_step(load_step)
        self.history.append(st)
        return ok

    def solveProblemOneCycle(self, load: List[LoadStep], dNdt: float) -> bool:
        any_d, st = self.problem.fatigue_cycle(load, dNdt)
        self.history.append(st)
        return any_d

    def solveProblemStatic(self, load: List[LoadStep], start_index: int = 0) -> int:
        """SolverFatigue::solveProblemStatic (solver_fatigue.h:244-275) with its halve-and-retry;
        returns the new start_index."""
        for i, step in enumerate(load):
            ok, st = self.problem.fatigue_static_step(step)
            st["step"] = i + start_index
            self.history.append(st)
            if not ok:
                raise LpmGpuError(ERR_CUTS, f"load step {i + start_index}")
            if self.dumpFile:
                self.problem.dump_write(self.dumpFile, i, self.ass.box, async_=True)
        self.problem.dump_flush()
        return start_index + len(load)

    def solveProblemCyclic(self, loadType: FatigueLoadType, n_interval: int, pt_groups) -> int:
        """SolverFatigue::solveProblemCyclic (solver_fatigue.h:183-218): one simulated cycle per
        pass, each standing for dN/dt real cycles, until the spectrum's cycle count is reached;
        the dump after each cycle is tagged with the cycle count N.  Returns N."""
        n_cycles = 0.5 * (len(self.load_spectrum) - 1)
        t, N = 0.0, 0
        while True:
            load_cycle = self.generateLoadCycle(loadType, N, n_interval, pt_groups)
            if self.t_mode == TimeMapMode.Linear:
                dNdt = func_dNdt_linear(self.tau)
            else:
                dNdt = func_dNdt_exponental(self.tau, t)
                t += 1
            self.solveProblemOneCycle(load_cycle, dNdt)
            N += int(dNdt)
            if self.dumpFile:
                self.problem.dump_write(self.dumpFile, N, self.ass.box, async_=True)
            if not N < n_cycles:
                break
        self.problem.dump_flush()
        return N
