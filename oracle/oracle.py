"""Test infrastructure (oracle): ctypes binding of the plain-C restatement in
oracle/lpm_oracle.c, plus helpers that run the reference's own build (oracle/_ref/lpm_ref).

Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import this
module.  It is the checker, never the product path.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liblpm_oracle.so")
REF_BIN = os.path.join(HERE, "_ref", "lpm_ref")
# the same driver built with SolverStaticGPU (lpm-cpp_b200/cpp/solver_static_gpu.h) in place of
# SolverStatic: the reference's Assembly and LoadStep code calling the device library
REF_GPU_BIN = os.path.join(HERE, "_ref", "lpm_ref_gpu")

LATTICES = {"sq2d": 0, "hex2d": 1, "sc3d": 2, "fcc3d": 3, "bcc3d": 4}
PTYPES = {"elastic": 0, "elastic_damage": 1, "j2": 2, "fatigue_hcf": 3}


class _Desc(C.Structure):
    _fields_ = [
        ("lattice", C.c_int), ("ptype", C.c_int), ("n", C.c_int),
        ("xyz", C.POINTER(C.c_double)), ("type", C.POINTER(C.c_int)),
        ("radius", C.c_double), ("plane_stress", C.c_int),
        ("E", C.c_double), ("mu", C.c_double), ("critical_bstrain", C.c_double),
        ("sigmay", C.c_double), ("xi", C.c_double), ("H", C.c_double), ("A", C.c_double),
        ("nonlocal_L", C.c_double), ("nonlocal_cutoff_ratio", C.c_double),
        ("undamaged_type", C.c_int), ("max_iter", C.c_int), ("tol_iter", C.c_double),
        ("cg_rtol", C.c_double), ("cg_atol", C.c_double), ("cg_maxit", C.c_longlong),
        ("bond_nb0", C.POINTER(C.c_int)), ("bond_nb1", C.POINTER(C.c_int)), ("bond_p2", C.POINTER(C.c_int)),
        ("tangent", C.c_int),
        ("k0", C.c_double), ("k1", C.c_double), ("comp_tensile_ratio", C.c_double), ("damage_threshold", C.c_double),
        ("fatigue_A", C.c_double), ("fatigue_B", C.c_double), ("fatigue_d", C.c_double),
        ("fatigue_limit_ratio", C.c_double),
        ("C11", C.c_double), ("C12", C.c_double), ("C44", C.c_double),
    ]


class _DispBC(C.Structure):
    _fields_ = [("ids", C.POINTER(C.c_int)), ("count", C.c_int), ("flag", C.c_int), ("step", C.c_double)]


class _ForceBC(C.Structure):
    _fields_ = [("ids", C.POINTER(C.c_int)), ("count", C.c_int),
                ("fx", C.c_double), ("fy", C.c_double), ("fz", C.c_double)]


class _LoadStep(C.Structure):
    _fields_ = [("disp", C.POINTER(_DispBC)), ("ndisp", C.c_int),
                ("force", C.POINTER(_ForceBC)), ("nforce", C.c_int)]


class _Stats(C.Structure):
    _fields_ = [("newton_solves", C.c_int), ("cg_iters", C.c_longlong), ("cuts", C.c_int),
                ("converged", C.c_int), ("reaction_norm", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.run(["make", "-s", "-C", HERE], check=True)
        L = C.CDLL(LIB_PATH)
        dp, ip, llp = C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_longlong)
        L.lpmo_generate.restype = C.c_long
        L.lpmo_generate.argtypes = [C.c_int, C.c_double, dp, dp, dp, C.c_long]
        L.lpmo_rmatrix.argtypes = [C.c_int, dp, dp]
        L.lpmo_create.restype = C.c_void_p
        L.lpmo_create.argtypes = [C.POINTER(_Desc)]
        L.lpmo_destroy.argtypes = [C.c_void_p]
        for f in ("lpmo_dim", "lpmo_nstate_var"):
            getattr(L, f).restype = C.c_int
            getattr(L, f).argtypes = [C.c_void_p]
        for f in ("lpmo_nbonds", "lpmo_nconn_total"):
            getattr(L, f).restype = C.c_long
            getattr(L, f).argtypes = [C.c_void_p]
        L.lpmo_nnz_upper.restype = C.c_longlong
        L.lpmo_nnz_upper.argtypes = [C.c_void_p]
        L.lpmo_get_bonds.argtypes = [C.c_void_p, ip, ip, ip]
        L.lpmo_get_conns.argtypes = [C.c_void_p, ip, ip, ip]
        for f in ("lpmo_update_geometry", "lpmo_update_force_state", "lpmo_update_state_var"):
            getattr(L, f).argtypes = [C.c_void_p]
        L.lpmo_update_rr.restype = C.c_double
        L.lpmo_update_rr.argtypes = [C.c_void_p]
        L.lpmo_assemble.argtypes = [C.c_void_p, C.c_int]
        L.lpmo_export_csr.argtypes = [C.c_void_p, llp, llp, llp, dp]
        L.lpmo_cg.restype = C.c_longlong
        L.lpmo_cg.argtypes = [C.c_void_p, dp]
        L.lpmo_apply_bc.argtypes = [C.c_void_p, C.POINTER(_LoadStep)]
        L.lpmo_solve_problem_step.restype = C.c_int
        L.lpmo_solve_problem_step.argtypes = [C.c_void_p, C.POINTER(_LoadStep), C.POINTER(_Stats)]
        L.lpmo_solve_load_step.restype = C.c_int
        L.lpmo_solve_load_step.argtypes = [C.c_void_p, C.POINTER(_LoadStep), C.POINTER(_Stats)]
        for f in ("lpmo_fatigue_solve_step", "lpmo_fatigue_static_step"):
            getattr(L, f).restype = C.c_int
            getattr(L, f).argtypes = [C.c_void_p, C.POINTER(_LoadStep), C.POINTER(_Stats)]
        L.lpmo_fatigue_update_damage.restype = C.c_int
        L.lpmo_fatigue_update_damage.argtypes = [C.c_void_p, C.c_double]
        L.lpmo_fatigue_cycle.restype = C.c_int
        L.lpmo_fatigue_cycle.argtypes = [C.c_void_p, C.POINTER(_LoadStep), C.c_int, C.c_double, C.POINTER(_Stats)]
        L.lpmo_read_state.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp, dp]
        L.lpmo_read_residual.argtypes = [C.c_void_p, dp]
        L.lpmo_set_xyz.argtypes = [C.c_void_p, dp]
        L.lpmo_get_bond_kntv.argtypes = [C.c_void_p, dp, dp]
        L.lpmo_set_bond_kntv.argtypes = [C.c_void_p, dp, dp]
        L.lpmo_set_bond_damage.argtypes = [C.c_void_p, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _llp(a):
    return a.ctypes.data_as(C.POINTER(C.c_longlong))


def rmatrix(flag: int, angles) -> np.ndarray:
    a = np.ascontiguousarray(angles, dtype=np.float64)
    R = np.zeros(9)
    lib().lpmo_rmatrix(flag, _dp(a), _dp(R))
    return R


def generate(lattice: str, radius: float, box, euler_flag=0, angles=(0.0, 0.0, 0.0)) -> np.ndarray:
    """Lattice generators of include/utilities.h:93-310 (restated)."""
    b = np.ascontiguousarray(box, dtype=np.float64)
    R = rmatrix(euler_flag, angles)
    n = lib().lpmo_generate(LATTICES[lattice], radius, _dp(b), _dp(R), None, 0)
    out = np.zeros((n, 3))
    lib().lpmo_generate(LATTICES[lattice], radius, _dp(b), _dp(R), _dp(out), n)
    return out


@dataclass
class Material:
    ptype: str = "elastic"
    plane_stress: bool = False
    E: float = 69e3
    mu: float = 0.3
    critical_bstrain: float = 1.0
    sigmay: float = 200.0
    xi: float = 0.0
    H: float = 0.0
    A: float = 0.0
    nonlocal_L: float = 0.0
    # ParticleElasticDamage (particle_elastic_damage.h:183-220)
    k0: float = 0.0
    k1: float = 1.0
    comp_tensile_ratio: float = 10.0
    damage_threshold: float = 1.0
    # ParticleFatigueHCF (particle_fatigue_hcf.h:163-205)
    fatigue_A: float = 0.0
    fatigue_B: float = 0.0
    fatigue_d: float = 0.0
    fatigue_limit_ratio: float = 1.108
    # setParticleProperty's (C11, C12, C44) overload; C11 > 0 takes it (particle_elastic.h:110-140)
    C11: float = 0.0
    C12: float = 0.0
    C44: float = 0.0


class _StepHolder:
    """Keeps the ctypes arrays of one load step alive."""

    def __init__(self, disp, force):
        self.keep = []
        nd, nf = len(disp), len(force)
        self.d = (_DispBC * max(nd, 1))()
        self.f = (_ForceBC * max(nf, 1))()
        for q, (ids, flag, step) in enumerate(disp):
            a = np.ascontiguousarray(ids, dtype=np.int32)
            self.keep.append(a)
            self.d[q] = _DispBC(_ip(a), len(a), int(flag), float(step))
        for q, (ids, fx, fy, fz) in enumerate(force):
            a = np.ascontiguousarray(ids, dtype=np.int32)
            self.keep.append(a)
            self.f[q] = _ForceBC(_ip(a), len(a), float(fx), float(fy), float(fz))
        self.s = _LoadStep(self.d, nd, self.f, nf)


class OracleProblem:
    """One problem in the C restatement.  ``disp`` entries are (ids, flag 0/1/2, step);
    ``force`` entries are (ids, fx, fy, fz)."""

    def __init__(self, lattice: str, radius: float, xyz: np.ndarray, mat: Material, types=None,
                 undamaged_type=-1, max_iter=30, tol_iter=1e-5, cg_rtol=1e-12, cg_atol=1e-12, cg_maxit=0,
                 nonlocal_cutoff_ratio=0.0, bonds=None, tangent=False):
        """bonds: optional (nb0, nb1, p2) lists as Assembly::readBond builds them; None runs the
        reference's bond search.  tangent: re-assemble K before every Newton solve."""
        self.xyz0 = np.ascontiguousarray(xyz, dtype=np.float64)
        self.n = len(self.xyz0)
        self.types = np.ascontiguousarray(types if types is not None else np.zeros(self.n), dtype=np.int32)
        d = _Desc()
        d.lattice, d.ptype, d.n = LATTICES[lattice], PTYPES[mat.ptype], self.n
        d.xyz, d.type = _dp(self.xyz0), _ip(self.types)
        d.radius, d.plane_stress = radius, int(mat.plane_stress)
        d.E, d.mu, d.critical_bstrain = mat.E, mat.mu, mat.critical_bstrain
        d.sigmay, d.xi, d.H, d.A = mat.sigmay, mat.xi, mat.H, mat.A
        d.nonlocal_L, d.nonlocal_cutoff_ratio = mat.nonlocal_L, nonlocal_cutoff_ratio
        d.undamaged_type, d.max_iter, d.tol_iter = undamaged_type, max_iter, tol_iter
        d.cg_rtol, d.cg_atol, d.cg_maxit = cg_rtol, cg_atol, cg_maxit
        d.tangent = int(bool(tangent))
        d.k0, d.k1, d.comp_tensile_ratio, d.damage_threshold = mat.k0, mat.k1, mat.comp_tensile_ratio, mat.damage_threshold
        d.fatigue_A, d.fatigue_B = getattr(mat, "fatigue_A", 0.0), getattr(mat, "fatigue_B", 0.0)
        d.fatigue_d, d.fatigue_limit_ratio = getattr(mat, "fatigue_d", 0.0), getattr(mat, "fatigue_limit_ratio", 1.108)
        d.C11, d.C12, d.C44 = getattr(mat, "C11", 0.0), getattr(mat, "C12", 0.0), getattr(mat, "C44", 0.0)
        if bonds is not None:
            self._bonds = [np.ascontiguousarray(a, dtype=np.int32) for a in bonds]
            d.bond_nb0, d.bond_nb1, d.bond_p2 = (_ip(a) for a in self._bonds)
        self._h = lib().lpmo_create(C.byref(d))
        self.dim = lib().lpmo_dim(self._h)
        self.nsv = lib().lpmo_nstate_var(self._h)

    def __del__(self):
        if getattr(self, "_h", None):
            lib().lpmo_destroy(self._h)
            self._h = None

    # ---- topology
    def bonds(self):
        L = lib()
        nb0 = np.zeros(self.n, np.int32)
        nb1 = np.zeros(self.n, np.int32)
        p2 = np.zeros(L.lpmo_nbonds(self._h), np.int32)
        L.lpmo_get_bonds(self._h, _ip(nb0), _ip(nb1), _ip(p2))
        return nb0, nb1, p2

    def conns(self):
        L = lib()
        nconn = np.zeros(self.n, np.int32)
        nlq = np.zeros(self.n, np.int32)
        cl = np.zeros(L.lpmo_nconn_total(self._h), np.int32)
        L.lpmo_get_conns(self._h, _ip(nconn), _ip(nlq), _ip(cl))
        return nconn, nlq, cl

    # ---- physics
    def update_geometry(self):
        lib().lpmo_update_geometry(self._h)

    def update_force_state(self):
        lib().lpmo_update_force_state(self._h)

    def update_state_var(self):
        lib().lpmo_update_state_var(self._h)

    def update_rr(self) -> float:
        return lib().lpmo_update_rr(self._h)

    def residual(self):
        r = np.zeros(self.dim * self.n)
        lib().lpmo_read_residual(self._h, _dp(r))
        return r

    def assemble(self, apply_bc=True):
        lib().lpmo_assemble(self._h, int(apply_bc))

    def export_csr(self):
        L = lib()
        nnz = L.lpmo_nnz_upper(self._h)
        Kp = np.zeros(self.n + 1, np.int64)
        IK = np.zeros(self.dim * self.n + 1, np.int64)
        JK = np.zeros(nnz, np.int64)
        K = np.zeros(nnz)
        L.lpmo_export_csr(self._h, _llp(Kp), _llp(IK), _llp(JK), _dp(K))
        return Kp, IK, JK, K

    def cg(self):
        disp = np.zeros(self.dim * self.n)
        it = lib().lpmo_cg(self._h, _dp(disp))
        return disp, it

    def apply_bc(self, disp=(), force=()):
        h = _StepHolder(disp, force)
        lib().lpmo_apply_bc(self._h, C.byref(h.s))

    def solve_load_step(self, disp=(), force=()):
        h = _StepHolder(disp, force)
        st = _Stats()
        ok = lib().lpmo_solve_load_step(self._h, C.byref(h.s), C.byref(st))
        return bool(ok), {"newton_solves": st.newton_solves, "cg_iters": st.cg_iters, "cuts": st.cuts,
                          "reaction_norm": st.reaction_norm}

    def set_xyz(self, xyz):
        a = np.ascontiguousarray(xyz, dtype=np.float64)
        lib().lpmo_set_xyz(self._h, _dp(a))

    # ---- SolverFatigue (include/solver_fatigue.h)
    @staticmethod
    def _stats(st):
        return {"newton_solves": st.newton_solves, "cg_iters": st.cg_iters, "cuts": st.cuts,
                "converged": bool(st.converged), "reaction_norm": st.reaction_norm}

    def fatigue_static_step(self, disp=(), force=()):
        """One entry of SolverFatigue::solveProblemStatic (solver_fatigue.h:244-275)."""
        h = _StepHolder(disp, force)
        st = _Stats()
        ok = lib().lpmo_fatigue_static_step(self._h, C.byref(h.s), C.byref(st))
        return bool(ok), self._stats(st)

    def fatigue_cycle(self, steps, dNdt):
        """SolverFatigue::solveProblemOneCycle (solver_fatigue.h:221-241); steps: [(disp, force)].
        Returns (any_damaged, stats) with stats["cuts"] = the steps that did not converge."""
        hs = [_StepHolder(d, f) for d, f in steps]
        arr = (_LoadStep * max(len(hs), 1))(*[h.s for h in hs])
        st = _Stats()
        any_d = lib().lpmo_fatigue_cycle(self._h, arr, len(hs), float(dNdt), C.byref(st))
        return bool(any_d), self._stats(st)

    def fatigue_update_damage(self, dNdt):
        return bool(lib().lpmo_fatigue_update_damage(self._h, float(dNdt)))

    def bond_kntv(self):
        nb = lib().lpmo_nbonds(self._h)
        kn, tv = np.zeros(nb), np.zeros(nb)
        lib().lpmo_get_bond_kntv(self._h, _dp(kn), _dp(tv))
        return kn, tv

    def set_bond_kntv(self, kn, tv):
        a, b = (np.ascontiguousarray(v, dtype=np.float64) for v in (kn, tv))
        lib().lpmo_set_bond_kntv(self._h, _dp(a), _dp(b))

    def set_bond_damage(self, bdamage):
        a = np.ascontiguousarray(bdamage, dtype=np.float64)
        lib().lpmo_set_bond_damage(self._h, _dp(a))

    def state(self):
        L = lib()
        n = self.n
        out = {"xyz": np.zeros((n, 3)), "pin": np.zeros((n, 3)), "stress": np.zeros((n, 6)),
               "damage": np.zeros(n), "damage_visual": np.zeros(n), "state_var": np.zeros((n, self.nsv)),
               "bdamage": np.zeros(L.lpmo_nbonds(self._h))}
        L.lpmo_read_state(self._h, *[_dp(out[k]) for k in ("xyz", "pin", "stress", "damage", "damage_visual",
                                                             "state_var", "bdamage")])
        return out


# ----------------------------------------------------------------------------- reference build
def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def run_ref(spec_text: str, outdir: str, threads: int = 1, timeout: float = 600.0, binary: str = REF_BIN,
            mkl_threads: int = 0) -> str:
    """Runs the reference's own build on a spec (see oracle/ref_driver.cpp); returns stdout.
    threads sets OMP_NUM_THREADS; mkl_threads > 0 sets MKL_NUM_THREADS, the team of the MKL
    stand-in's sparse product and CG loops (otherwise it follows OMP_NUM_THREADS)."""
    os.makedirs(outdir, exist_ok=True)
    path = os.path.join(outdir, "spec.txt")
    with open(path, "w") as f:
        f.write(spec_text + f"\nout {outdir}\n")
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    env.pop("MKL_NUM_THREADS", None)
    if mkl_threads > 0:
        env["MKL_NUM_THREADS"] = str(int(mkl_threads))
    r = subprocess.run([binary, path], env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"{os.path.basename(binary)} failed ({r.returncode}): {r.stderr[-2000:]}")
    return r.stdout


def read_ref_steps(outdir: str):
    rows = []
    with open(os.path.join(outdir, "steps.txt")) as f:
        for line in f:
            if line.startswith("#"):
                continue
            t = line.split()
            rows.append({"step": int(t[0]), "newton_solves": int(t[1]), "cg_iters": int(t[2]),
                         "wall_s": float(t[3]), "spmv_s": float(t[4]), "cg_s": float(t[5]),
                         "create_s": float(t[6]), "cuts": int(t[7]), "reaction_norm": float(t[8])})
    return rows


def read_bin(outdir: str, name: str, dtype) -> np.ndarray:
    return np.fromfile(os.path.join(outdir, name), dtype=dtype)


def write_bond_file(path: str, nb0, nb1, p2):
    """Bond lists in the reference's text format, one "id layer p1 p2" line per bond in
    (particle, layer-0 then layer-1) order, as Assembly::writeBond prints them (assembly.h:269-283)."""
    nb0, nb1, p2 = (np.asarray(a, dtype=np.int64) for a in (nb0, nb1, p2))
    nb = nb0 + nb1
    p1 = np.repeat(np.arange(len(nb)), nb)
    start = np.concatenate([[0], np.cumsum(nb)[:-1]])
    layer = (np.arange(len(p2)) - np.repeat(start, nb) >= np.repeat(nb0, nb)).astype(np.int64)
    rows = np.stack([np.arange(len(p2)), layer, p1, p2], axis=1)
    np.savetxt(path, rows, fmt="%d")


def write_ref_spec(case, outdir: str, steps=None, max_iter=None, tol_iter=None, cg_tol=None, cg_maxit_cap=0,
                   dump_k=(), loop="step", use_generator=True, tangent=False, solver="cg", solve_threads=0) -> str:
    """Spec text for oracle/_ref/lpm_ref describing a product-side ``Case`` (duck-typed):
    groups and particle types are passed as raw int32 id files so both sides see the same sets.
    With use_generator the reference generates the lattice itself (its ids must then equal
    case.xyz, which the tests check); otherwise case.xyz is passed as a coordinate file."""
    os.makedirs(outdir, exist_ok=True)
    lat = {0: "sq2d", 1: "hex2d", 2: "sc3d", 3: "fcc3d", 4: "bcc3d"}[int(case.lattice)]
    m = case.material
    lines = [f"lattice {lat}", f"radius {case.radius!r}", "box " + " ".join(repr(float(v)) for v in case.box),
             f"euler {case.euler[0]} " + " ".join(repr(float(a)) for a in case.euler[1]),
             f"ptype {({2: 'j2', 1: 'elastic_damage', 3: 'fatigue_hcf'}).get(int(case.ptype), 'elastic')}",
             f"plane_stress {int(m.plane_stress)}",
             f"cij {getattr(m, 'C11', 0.0)!r} {getattr(m, 'C12', 0.0)!r} {getattr(m, 'C44', 0.0)!r}",
             f"hcf {getattr(m, 'fatigue_A', 0.0)!r} {getattr(m, 'fatigue_B', 0.0)!r} {getattr(m, 'fatigue_d', 0.0)!r} "
             f"{getattr(m, 'damage_threshold', 1.0)!r} {getattr(m, 'fatigue_limit_ratio', 1.108)!r}",
             f"edamage {getattr(m, 'k0', 0.0)!r} {getattr(m, 'k1', 1.0)!r} {getattr(m, 'comp_tensile_ratio', 10.0)!r} "
             f"{getattr(m, 'damage_threshold', 1.0)!r}",
             f"nonlocal_cutoff_ratio {float(getattr(case, 'nonlocal_cutoff_ratio', 0.0))!r}",
             f"E {m.E!r}", f"mu {m.mu!r}", f"critical_bstrain {m.critical_bstrain!r}",
             f"j2 {m.sigmay!r} {m.xi!r} {m.H!r} {m.A!r}", f"nonlocal_L {m.nonlocal_L!r}",
             f"undamaged_type {case.undamaged_type}",
             f"max_iter {case.max_iter if max_iter is None else max_iter}",
             f"tol_iter {(case.tol_iter if tol_iter is None else tol_iter)!r}", f"loop {loop}"]
    if cg_maxit_cap:
        lines.append(f"cg_maxit_cap {int(cg_maxit_cap)}")
    if solve_threads:
        lines.append(f"solve_threads {int(solve_threads)}")
    if tangent:
        lines.append("tangent 1")
    if solver != "cg":
        lines.append(f"solver {solver}")
    if cg_tol is not None:
        lines.append(f"cg_tol {cg_tol[0]!r} {cg_tol[1]!r}")
    if not use_generator or lat == "bcc3d":
        p = os.path.join(outdir, "xyz_in.f64")
        np.ascontiguousarray(case.xyz, dtype=np.float64).tofile(p)
        lines.append(f"xyz_file {p}")
    if getattr(case, "bonds", None) is not None:
        p = os.path.join(outdir, "bonds_in.txt")
        write_bond_file(p, *case.bonds)
        lines.append(f"bondfile {p}")
    if getattr(case, "bond_props", None) is not None:
        p = os.path.join(outdir, "bondprops_in.f64")
        np.concatenate([np.asarray(a, dtype=np.float64) for a in case.bond_props]).tofile(p)
        lines.append(f"bondprops {p}")
    p = os.path.join(outdir, "types_in.i32")
    np.ascontiguousarray(case.types, dtype=np.int32).tofile(p)
    lines.append(f"typefile {p}")
    for name, ids in case.groups.items():
        p = os.path.join(outdir, f"group_{name}.i32")
        np.ascontiguousarray(ids, dtype=np.int32).tofile(p)
        lines.append(f"groupfile {name} {p}")
    nsteps = len(case.steps) if steps is None else steps
    lines.append(f"steps {nsteps}")
    for s in range(nsteps):
        disp, force = case.steps[s % len(case.steps)]
        for g, flag, v in disp:
            lines.append(f"dispbc {g} {flag} {float(v)!r} {s} {s + 1}")
        for g, fx, fy, fz in force:
            lines.append(f"forcebc {g} {float(fx)!r} {float(fy)!r} {float(fz)!r} {s} {s + 1}")
    for k in dump_k:
        lines.append(f"dumpK {int(k)}")
    fat = getattr(case, "meta", {}).get("fatigue")
    if fat is not None:
        p = os.path.join(outdir, "fatigue_load.txt")
        with open(p, "w") as f:
            f.write("\n".join(repr(float(v)) for v in fat["spectrum"]) + "\n")
        lines.append(f"fatigue {fat['load_type']} {int(fat['n_interval'])} {fat['tmode']} {float(fat['tau'])!r}")
        lines.append("fatigue_groups " + " ".join(fat["groups"]))
        lines.append(f"fatigue_load {p}")
    return "\n".join(lines) + "\n"
